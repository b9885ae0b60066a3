// Matching-cost DSI writers, banded: Birchfield-Tomasi (tdvision/birchfieldcost.cu:14-59),
// window SSD (ssd.cu:15-50) and un-centred NCC (crosscorrelation.cu:11-49).
//
// One CTA owns a tile of kTX x kTY pixels and all D disparities of them.
//   * Staging: the rows the tile's windows touch are read once, clamped to
//     each image's own edges and multiplied by its scale exactly as the
//     per-cell reference fetch does, into shared memory: raw bands for SSD /
//     NCC; for BT the per-pixel left terms (I, min, max of I and its two
//     half-sums) and the per-column right terms, which depend on x - d only.
//     NCC also stages the window sums of l^2 (per pixel) and r^2 (per column
//     x - d), summed in the reference's tap order.
//   * Compute: warp lanes are disparities (32 per warp, or 8 / 16 with two
//     or four pixel groups per warp when D is small) and each thread walks
//     P consecutive pixels, so the right-band reads of a warp are 32
//     consecutive words (no bank conflict) and the left-band reads are
//     broadcasts.  Across the P pixels of a thread the tap values of one
//     window row depend only on the column, so each squared difference
//     (SSD) or product (NCC) is formed once per column and then accumulated
//     into every pixel whose window holds it -- in each pixel's own row-major
//     tap order, so every cell is rounded exactly as the reference's loop
//     rounds it.
//   * Stores: a warp writes the D-contiguous run of one pixel, a full
//     128-byte line per instruction in either DSI layout.
// Cells with x - d < 0 are +INF (the reference's range rule).
#include <cuda_runtime.h>
#include <math_constants.h>

#include <atomic>
#include <cstdint>

#include "gauss5.cuh"
#include "tdv_internal.hpp"

namespace tdv {

namespace {

constexpr int kTX = 64;           // tile width (pixels)
constexpr int kTY = 4;            // tile height (rows)
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxBandBytes = 100 * 1024;

__device__ __forceinline__ float fetch(const ImgArg& im, int x, int y) {
    x = min(max(x, 0), im.W - 1);
    y = min(max(y, 0), im.H - 1);
    const size_t o = (size_t)y * im.pitch + x;
    if (im.u8) return __fmul_rn((float)((const uint8_t*)im.ptr)[o], im.scale);
    return __fmul_rn(((const float*)im.ptr)[o], im.scale);
}

struct Geom {
    int D, Dw, G;      // disparities; lanes per pixel group (8, 16 or 32); groups per warp
    int rbw;           // right-band width: columns x0-(D-1)-r .. x0+kTX-1+r
    int lbw;           // left-band width: columns x0-r .. x0+kTX-1+r, padded to 4 floats
};

__host__ __device__ constexpr int left_band_width(int r) { return kTX + ((2 * r + 3) & ~3); }

// Shared-memory layout (floats) of one tile.
template <int KIND, int R>
struct Band {
    static constexpr int kRows = kTY + 2 * R;
    __host__ __device__ static int rband(const Geom& g) { return KIND == TDV_COST_BT ? 3 * kTX * kTY : kRows * g.lbw; }
    // NCC window sums: LS per tile pixel, RS per (row, column x - d)
    __host__ __device__ static int ls(const Geom& g) { return rband(g) + kRows * g.rbw; }
    __host__ __device__ static int rs(const Geom& g) { return ls(g) + kTX * kTY; }
    __host__ __device__ static int floats(const Geom& g) {
        if (KIND == TDV_COST_BT) return 3 * kTX * kTY + 3 * kTY * (kTX + g.D - 1);
        if (KIND == TDV_COST_SSD) return kRows * g.lbw + kRows * g.rbw;
        return kRows * g.lbw + kRows * g.rbw + kTX * kTY + kTY * (kTX + g.D - 1);
    }
    // With the Gaussian fused: BT first builds filtered bands of the left
    // (kTX + 2 columns) and right (kTX + D + 1 columns) rows; every kind needs
    // the raw rows with a 2-pixel halo and their row pass as scratch.
    __host__ __device__ static int fl_band(const Geom& g) { return floats(g); }
    __host__ __device__ static int fr_band(const Geom& g) { return fl_band(g) + kTY * (kTX + 2); }
    __host__ __device__ static int widest(const Geom& g) {
        return KIND == TDV_COST_BT ? kTX + g.D + 1 : (g.lbw > g.rbw ? g.lbw : g.rbw);
    }
    __host__ __device__ static int scratch(const Geom& g) {
        return KIND == TDV_COST_BT ? fr_band(g) + kTY * (kTX + g.D + 1) : floats(g);
    }
    __host__ __device__ static int floats_filtered(const Geom& g) {
        const int rows = (KIND == TDV_COST_BT ? kTY : kRows) + 4, w = widest(g);
        return scratch(g) + rows * (w + 4) + rows * w;
    }
};

// BT terms of one sample: I, min and max of {I, (I + I[-1]) / 2, (I + I[+1]) / 2}.
__device__ __forceinline__ void bt_terms(const ImgArg& im, int x, int y, float& I, float& mi, float& ma) {
    I = fetch(im, x, y);
    const float a = __fmul_rn(0.5f, __fadd_rn(I, fetch(im, x - 1, y)));
    const float b = __fmul_rn(0.5f, __fadd_rn(I, fetch(im, x + 1, y)));
    mi = fminf(a, fminf(b, I));
    ma = fmaxf(a, fmaxf(b, I));
}

// band[row * bw + col] = G(clamp(c0 + col), clamp(r0 + row)) for the 5x5
// Gaussian G of the image with replicated borders (the pre-filter kernel's
// values, bit for bit): the raw rows the clamped range needs, with a 2-pixel
// halo, then the row pass, then the column pass, in that kernel's order.
__device__ void gauss_band(const ImgArg& im, int c0, int ncols, int r0, int nrows, float* band, int bw,
                           float* scratch) {
    const int tid = threadIdx.x;
    const int c_lo = min(max(c0, 0), im.W - 1), c_hi = min(max(c0 + ncols - 1, 0), im.W - 1);
    const int r_lo = min(max(r0, 0), im.H - 1), r_hi = min(max(r0 + nrows - 1, 0), im.H - 1);
    const int nc = c_hi - c_lo + 1, nr = r_hi - r_lo + 1;
    float* raw = scratch;                   // [nr + 4][nc + 4]
    float* rp = scratch + (nr + 4) * (nc + 4);  // [nr + 4][nc]
    for (int i = tid; i < (nr + 4) * (nc + 4); i += kThreads) {
        const int row = i / (nc + 4), col = i - row * (nc + 4);
        raw[i] = fetch(im, c_lo - 2 + col, r_lo - 2 + row);
    }
    __syncthreads();
    for (int i = tid; i < (nr + 4) * nc; i += kThreads) {
        const int row = i / nc, col = i - row * nc;
        const float* t = raw + row * (nc + 4) + col;
        rp[i] = gauss5(t[0], t[1], t[2], t[3], t[4]);
    }
    __syncthreads();
    for (int i = tid; i < nrows * ncols; i += kThreads) {
        const int row = i / ncols, col = i - row * ncols;
        const int cc = min(max(c0 + col, 0), im.W - 1) - c_lo, rr = min(max(r0 + row, 0), im.H - 1) - r_lo;
        const float* t = rp + rr * nc + cc;
        band[row * bw + col] = gauss5(t[0], t[nc], t[2 * nc], t[3 * nc], t[4 * nc]);
    }
    __syncthreads();
}

// BT terms from a band of (filtered) samples: b[0], b[1], b[2] are the
// samples at x - 1, x, x + 1.
__device__ __forceinline__ void bt_terms_band(const float* b, float& I, float& mi, float& ma) {
    I = b[1];
    const float a = __fmul_rn(0.5f, __fadd_rn(I, b[0]));
    const float c = __fmul_rn(0.5f, __fadd_rn(I, b[2]));
    mi = fminf(a, fminf(c, I));
    ma = fmaxf(a, fmaxf(c, I));
}

template <int R>
__device__ void ncc_sums(const Geom& g, float* sm);

template <int KIND, int R>
__device__ void stage_plain(const ImgArg& L, const ImgArg& Rim, const Geom& g, int x0, int y0, float* sm) {
    using B = Band<KIND, R>;
    const int tid = threadIdx.x;
    if (KIND == TDV_COST_BT) {
        float* lt = sm;                  // [3][kTY][kTX]
        float* rt = sm + B::rband(g);    // [3][kTY][kTX + D - 1]
        for (int i = tid; i < kTX * kTY; i += kThreads) {
            const int row = i / kTX, col = i - row * kTX;
            float I, mi, ma;
            bt_terms(L, x0 + col, y0 + row, I, mi, ma);
            lt[i] = I;
            lt[kTX * kTY + i] = mi;
            lt[2 * kTX * kTY + i] = ma;
        }
        const int rw = kTX + g.D - 1, n = rw * kTY;
        float2* rmm = reinterpret_cast<float2*>(rt + n);  // (min, max) pairs, 8-byte aligned
        for (int i = tid; i < n; i += kThreads) {
            const int row = i / rw, col = i - row * rw;
            float I, mi, ma;
            bt_terms(Rim, x0 - (g.D - 1) + col, y0 + row, I, mi, ma);
            rt[i] = I;
            rmm[i] = make_float2(mi, ma);
        }
        return;
    }
    float* lb = sm;                       // [kRows][lbw], column x0 - R at index 0
    float* rb = sm + B::rband(g);         // [kRows][rbw], column x0 - (D-1) - R at index 0
    for (int i = tid; i < B::kRows * g.lbw; i += kThreads) {
        const int row = i / g.lbw, col = i - row * g.lbw;
        lb[i] = fetch(L, x0 - R + col, y0 - R + row);
    }
    for (int i = tid; i < B::kRows * g.rbw; i += kThreads) {
        const int row = i / g.rbw, col = i - row * g.rbw;
        rb[i] = fetch(Rim, x0 - (g.D - 1) - R + col, y0 - R + row);
    }
    if (KIND != TDV_COST_NCC) return;
    __syncthreads();
    ncc_sums<R>(g, sm);
}

// NCC: window sums of squares in the reference's tap order (rows, then
// columns), LS per tile pixel from the left band, RS per column x - d.
template <int R>
__device__ void ncc_sums(const Geom& g, float* sm) {
    using B = Band<TDV_COST_NCC, R>;
    const int tid = threadIdx.x;
    const float* lb = sm;
    const float* rb = sm + B::rband(g);
    float* ls = sm + B::ls(g);
    float* rs = sm + B::rs(g);
    for (int i = tid; i < kTX * kTY; i += kThreads) {
        const int row = i / kTX, col = i - row * kTX;
        float s = 0.0f;
        for (int a = 0; a <= 2 * R; a++)
            for (int b = 0; b <= 2 * R; b++) {
                const float v = lb[(row + a) * g.lbw + col + b];
                s = __fadd_rn(s, __fmul_rn(v, v));
            }
        ls[i] = s;
    }
    const int rw = kTX + g.D - 1;
    for (int i = tid; i < rw * kTY; i += kThreads) {
        const int row = i / rw, col = i - row * rw;
        float s = 0.0f;
        for (int a = 0; a <= 2 * R; a++)
            for (int b = 0; b <= 2 * R; b++) {
                const float v = rb[(row + a) * g.rbw + col + b];
                s = __fadd_rn(s, __fmul_rn(v, v));
            }
        rs[i] = s;
    }
}

// Fills the tile's bands (and, when FILT, writes the filtered left samples of
// the tile's own pixels to fl_out, W x H dense).
template <int KIND, int R, bool FILT>
__device__ void stage(const ImgArg& L, const ImgArg& Rim, const Geom& g, int x0, int y0, float* sm, int W, int H,
                      float* fl_out) {
    using B = Band<KIND, R>;
    const int tid = threadIdx.x;
    if (FILT && KIND == TDV_COST_BT) {
        float* fl = sm + B::fl_band(g);     // [kTY][kTX + 2]: columns x0 - 1 .. x0 + kTX
        float* fr = sm + B::fr_band(g);     // [kTY][kTX + D + 1]: columns x0 - D .. x0 + kTX
        float* scr = sm + B::scratch(g);
        gauss_band(L, x0 - 1, kTX + 2, y0, kTY, fl, kTX + 2, scr);
        gauss_band(Rim, x0 - g.D, kTX + g.D + 1, y0, kTY, fr, kTX + g.D + 1, scr);
        float* lt = sm;
        float* rt = sm + B::rband(g);
        for (int i = tid; i < kTX * kTY; i += kThreads) {
            const int row = i / kTX, col = i - row * kTX;
            float I, mi, ma;
            bt_terms_band(fl + row * (kTX + 2) + col, I, mi, ma);
            lt[i] = I;
            lt[kTX * kTY + i] = mi;
            lt[2 * kTX * kTY + i] = ma;
            const int x = x0 + col, y = y0 + row;
            if (fl_out && x < W && y < H) fl_out[(size_t)y * W + x] = I;
        }
        const int rw = kTX + g.D - 1, n = rw * kTY;
        float2* rmm = reinterpret_cast<float2*>(rt + n);
        for (int i = tid; i < n; i += kThreads) {
            const int row = i / rw, col = i - row * rw;
            float I, mi, ma;
            bt_terms_band(fr + row * (kTX + g.D + 1) + col, I, mi, ma);
            rt[i] = I;
            rmm[i] = make_float2(mi, ma);
        }
        return;
    }
    if (FILT) {
        float* lb = sm;
        float* rb = sm + B::rband(g);
        float* scr = sm + B::scratch(g);
        gauss_band(L, x0 - R, g.lbw, y0 - R, B::kRows, lb, g.lbw, scr);
        gauss_band(Rim, x0 - (g.D - 1) - R, g.rbw, y0 - R, B::kRows, rb, g.rbw, scr);
        if (fl_out)
            for (int i = tid; i < kTX * kTY; i += kThreads) {
                const int row = i / kTX, col = i - row * kTX;
                const int x = x0 + col, y = y0 + row;
                if (x < W && y < H) fl_out[(size_t)y * W + x] = lb[(row + R) * g.lbw + col + R];
            }
        if (KIND == TDV_COST_NCC) ncc_sums<R>(g, sm);
        return;
    }
    stage_plain<KIND, R>(L, Rim, g, x0, y0, sm);
}

template <int KIND, int R, int P, bool FILT>
__global__ void __launch_bounds__(kThreads) cost_band_kernel(ImgArg L, ImgArg Rim, VolArg out, Geom g,
                                                             int tiles_x, float* fl_out) {
    extern __shared__ __align__(16) float sm[];
    using B = Band<KIND, R>;
    const int x0 = (blockIdx.x % tiles_x) * kTX, y0 = (blockIdx.x / tiles_x) * kTY;
    stage<KIND, R, FILT>(L, Rim, g, x0, y0, sm, out.W, out.H, fl_out);
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int D = g.D, W = out.W, H = out.H;
    const int sub = lane / g.Dw, dl = lane - sub * g.Dw;
    const int span = P * g.G;                   // pixels of one work item
    const int groups = kTX / span;
    const int chunks = (D + g.Dw - 1) / g.Dw;
    const int items = kTY * groups * chunks;
    float* const outp = (float*)out.ptr;

    if (KIND == TDV_COST_BT) {
        // BT: a work item is P pixels of one row over every disparity chunk,
        // so each pixel's left terms are read from shared memory once
        const float* lt = sm;
        const float* rt = sm + B::rband(g);
        const int n = (kTX + D - 1) * kTY;
        for (int it = warp; it < kTY * groups; it += kWarps) {
            const int grp = it % groups, row = it / groups;
            const int y = y0 + row;
            const int xs = x0 + grp * span + sub * P;
            float lI[P], lImi[P], lIma[P];
#pragma unroll
            for (int p = 0; p < P; p++) {
                const int li = row * kTX + (xs + p - x0);
                lI[p] = lt[li];
                lImi[p] = lt[kTX * kTY + li];
                lIma[p] = lt[2 * kTX * kTY + li];
            }
            const float2* rmm = reinterpret_cast<const float2*>(rt + n);
            const bool rows_in = y < H && xs + P <= W;
            for (int chunk = 0; chunk < chunks; chunk++) {
                const int d = chunk * g.Dw + dl;
                const bool dok = d < D;
                const int de = dok ? d : D - 1;
                const int r0 = row * (kTX + D - 1) + (xs - de) - (x0 - (D - 1));
                const long long oi = y * out.sy + d + xs * out.sx;
                float v[P];
#pragma unroll
                for (int p = 0; p < P; p++) {
                    const float rI = rt[r0 + p];
                    const float2 mm = rmm[r0 + p];
                    const float a = fmaxf(0.0f, fmaxf(__fsub_rn(lI[p], mm.y), __fsub_rn(mm.x, lI[p])));
                    const float b = fmaxf(0.0f, fmaxf(__fsub_rn(rI, lIma[p]), __fsub_rn(lImi[p], rI)));
                    v[p] = __fadd_rn(0.0f, fminf(a, b));
                }
                if (out.u16) {
                    // 16-bit DSI (integer intensities only): half-units, +INF as 0xFFFF
                    uint16_t* const op = (uint16_t*)out.ptr + oi;
                    if (dok && rows_in && xs - d >= 0) {
#pragma unroll
                        for (int p = 0; p < P; p++) op[p * out.sx] = (uint16_t)__float2uint_rn(__fmul_rn(v[p], 2.0f));
                    } else if (dok && y < H) {
#pragma unroll
                        for (int p = 0; p < P; p++) {
                            const int x = xs + p;
                            if (x < W)
                                op[p * out.sx] = (x - d < 0) ? (uint16_t)0xFFFFu
                                                             : (uint16_t)__float2uint_rn(__fmul_rn(v[p], 2.0f));
                        }
                    }
                } else if (dok && rows_in && xs - d >= 0) {
                    // all P cells in the image and in range: plain stores
                    float* const op = outp + oi;
#pragma unroll
                    for (int p = 0; p < P; p++) op[p * out.sx] = v[p];
                } else if (dok && y < H) {
                    float* const op = outp + oi;
#pragma unroll
                    for (int p = 0; p < P; p++) {
                        const int x = xs + p;
                        if (x < W) op[p * out.sx] = (x - d < 0) ? CUDART_INF_F : v[p];
                    }
                }
            }
        }
        return;
    }

    if constexpr (KIND != TDV_COST_BT) {
        for (int it = warp; it < items; it += kWarps) {
            const int chunk = it % chunks;
            const int rest = it / chunks;
            const int grp = rest % groups, row = rest / groups;
            const int y = y0 + row;
            const int xs = x0 + grp * span + sub * P;   // first pixel of this thread
            const int d = chunk * g.Dw + dl;
            const bool dok = d < D;
            const int de = dok ? d : D - 1;             // lanes past D read in-band columns, store nothing
            float v[P];
            {
                constexpr int NJ = P + 2 * R;
                float acc[P];
    #pragma unroll
                for (int p = 0; p < P; p++) acc[p] = 0.0f;
                const float* lb = sm + (size_t)row * g.lbw + (xs - x0);
                const float* rb = sm + B::rband(g) + (size_t)row * g.rbw + (xs - de) - (x0 - (D - 1));
                constexpr int NJ4 = (NJ + 3) & ~3;
    #pragma unroll 1
                for (int a = 0; a <= 2 * R; a++) {
                    // the left window is the same for every lane: 128-bit
                    // broadcast reads (the row start is a multiple of 16 floats
                    // into a row padded to 4)
                    float lw[NJ4];
                    const float4* l4 = reinterpret_cast<const float4*>(lb + a * g.lbw);
    #pragma unroll
                    for (int q = 0; q < NJ4 / 4; q++) {
                        const float4 f = l4[q];
                        lw[4 * q] = f.x;
                        lw[4 * q + 1] = f.y;
                        lw[4 * q + 2] = f.z;
                        lw[4 * q + 3] = f.w;
                    }
                    float t[NJ];
    #pragma unroll
                    for (int j = 0; j < NJ; j++) {
                        const float lv = lw[j], rv = rb[a * g.rbw + j];
                        if (KIND == TDV_COST_SSD) {
                            const float df = __fsub_rn(lv, rv);
                            t[j] = __fmul_rn(df, df);
                        } else {
                            t[j] = __fmul_rn(lv, rv);
                        }
                    }
    #pragma unroll
                    for (int b = 0; b <= 2 * R; b++)
    #pragma unroll
                        for (int p = 0; p < P; p++) acc[p] = __fadd_rn(acc[p], t[p + b]);
                }
                if (KIND == TDV_COST_SSD) {
    #pragma unroll
                    for (int p = 0; p < P; p++) v[p] = acc[p];
                } else {
                    const float* ls = sm + B::ls(g) + row * kTX + (xs - x0);
                    const float* rs = sm + B::rs(g) + row * (kTX + D - 1) + (xs - de) - (x0 - (D - 1));
    #pragma unroll
                    for (int p = 0; p < P; p++)
                        v[p] = __fsub_rn(1.0f, __fdiv_rn(acc[p], __fsqrt_rn(__fmul_rn(ls[p], rs[p]))));
                }
            }
            if (!dok || y >= H) continue;
    #pragma unroll
            for (int p = 0; p < P; p++) {
                const int x = xs + p;
                if (x < W) outp[x * out.sx + y * out.sy + d] = (x - d < 0) ? CUDART_INF_F : v[p];
            }
        }
    }
}

// Bands above 48 KB need the kernel's dynamic shared-memory limit raised, an
// attribute of the function on each device: raised once per device (bit d of
// `opted`; devices past 63 set it on every launch).
template <typename Kern>
cudaError_t opt_in_once(Kern k, std::atomic<unsigned long long>& opted) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (bit && (opted.load() & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxBandBytes);
    if (e == cudaSuccess && bit) opted.fetch_or(bit);
    return e;
}

// Order-preserving key of a window SSD for the argmin.  An SSD is a sum of
// squares from +0, so it is +0, positive, +INF or NaN: its bits order the
// finite values, and clamping at the bits of +INF puts NaN and +INF on one
// key above every finite cost (the reference's `v < best` with best starting
// at +INF never takes either; when no cost is finite the lowest d, 0, wins
// the tie).  Cells outside the range keep the initial key 0xFFFFFFFF.
__device__ __forceinline__ uint32_t ssd_key(float v) { return min(__float_as_uint(v), 0x7F800000u); }

// FastWTA (tdvision/fastwta.cu:32-53): the window SSD of the banded kernel
// with the argmin over d fused in, no DSI.  A lane keeps the best (key, d)
// of its own disparities over the chunks (strict <, so its lowest d wins a
// tie), then the lanes of a pixel group merge by (key, d) -- the lowest d
// among the smallest costs, d = 0 when no cost is finite, as the reference's
// scan gives.  Eight pixels per thread (half the SSD kernel's sixteen) keep
// the per-pixel best keys within a register budget that fits four blocks per
// SM.
template <int R, int P>
__global__ void __launch_bounds__(kThreads) fastwta_band_kernel(ImgArg L, ImgArg Rim, int W, int H, Geom g,
                                                                int tiles_x, uint16_t* disp, float* disp_norm) {
    extern __shared__ __align__(16) float sm[];
    using B = Band<TDV_COST_SSD, R>;
    const int x0 = (blockIdx.x % tiles_x) * kTX, y0 = (blockIdx.x / tiles_x) * kTY;
    stage<TDV_COST_SSD, R, false>(L, Rim, g, x0, y0, sm, W, H, nullptr);
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int D = g.D;
    const int sub = lane / g.Dw, dl = lane - sub * g.Dw;
    const int span = P * g.G;
    const int groups = kTX / span;
    const int chunks = (D + g.Dw - 1) / g.Dw;
    constexpr int NJ = P + 2 * R;
    constexpr int NJ4 = (NJ + 3) & ~3;

    for (int it = warp; it < kTY * groups; it += kWarps) {
        const int grp = it % groups, row = it / groups;
        const int y = y0 + row;
        const int xs = x0 + grp * span + sub * P;
        uint32_t bk[P];
        int bd[P];
#pragma unroll
        for (int p = 0; p < P; p++) {
            bk[p] = 0xFFFFFFFFu;
            bd[p] = dl;
        }
        for (int chunk = 0; chunk < chunks; chunk++) {
            const int d = chunk * g.Dw + dl;
            const bool dok = d < D;
            const int de = dok ? d : D - 1;
            float acc[P];
#pragma unroll
            for (int p = 0; p < P; p++) acc[p] = 0.0f;
            const float* lb = sm + (size_t)row * g.lbw + (xs - x0);
            const float* rb = sm + B::rband(g) + (size_t)row * g.rbw + (xs - de) - (x0 - (D - 1));
#pragma unroll 1
            for (int a = 0; a <= 2 * R; a++) {
                float lw[NJ4];
                const float4* l4 = reinterpret_cast<const float4*>(lb + a * g.lbw);
#pragma unroll
                for (int q = 0; q < NJ4 / 4; q++) {
                    const float4 f = l4[q];
                    lw[4 * q] = f.x;
                    lw[4 * q + 1] = f.y;
                    lw[4 * q + 2] = f.z;
                    lw[4 * q + 3] = f.w;
                }
                float t[NJ];
#pragma unroll
                for (int j = 0; j < NJ; j++) {
                    const float df = __fsub_rn(lw[j], rb[a * g.rbw + j]);
                    t[j] = __fmul_rn(df, df);
                }
#pragma unroll
                for (int b = 0; b <= 2 * R; b++)
#pragma unroll
                    for (int p = 0; p < P; p++) acc[p] = __fadd_rn(acc[p], t[p + b]);
            }
            if (dok && xs - d >= 0) {  // every cell of the chunk in range
#pragma unroll
                for (int p = 0; p < P; p++) {
                    const uint32_t key = ssd_key(acc[p]);
                    if (key < bk[p]) {
                        bk[p] = key;
                        bd[p] = d;
                    }
                }
            } else if (dok) {
#pragma unroll
                for (int p = 0; p < P; p++) {
                    const uint32_t key = ssd_key(acc[p]);
                    if (xs + p - d >= 0 && key < bk[p]) {
                        bk[p] = key;
                        bd[p] = d;
                    }
                }
            }
        }
#pragma unroll
        for (int p = 0; p < P; p++) {
            uint32_t k = bk[p];
            int dd = bd[p];
            if (g.Dw == 32) {
                // the warp is one pixel group: the smallest key, then the
                // lowest d among the lanes holding it
                k = __reduce_min_sync(0xFFFFFFFFu, k);
                dd = (int)__reduce_min_sync(0xFFFFFFFFu, bk[p] == k ? (unsigned)dd : 0x7FFFFFFFu);
            } else {
                for (int off = g.Dw >> 1; off > 0; off >>= 1) {
                    const uint32_t ok = __shfl_xor_sync(0xFFFFFFFFu, k, off);
                    const int od = __shfl_xor_sync(0xFFFFFFFFu, dd, off);
                    if (ok < k || (ok == k && od < dd)) {
                        k = ok;
                        dd = od;
                    }
                }
            }
            const int x = xs + p;
            if (dl == 0 && x < W && y < H) {
                const size_t o = (size_t)y * W + x;
                if (disp) disp[o] = (uint16_t)dd;
                if (disp_norm) disp_norm[o] = __fdiv_rn((float)dd, (float)D);
            }
        }
    }
}

template <int R>
cudaError_t launch_fastwta_r(const ImgArg& L, const ImgArg& Rim, const Geom& g, uint16_t* disp, float* disp_norm,
                             cudaStream_t st) {
    const int bytes = Band<TDV_COST_SSD, R>::floats(g) * 4;
    auto k = fastwta_band_kernel<R, 8>;
    static std::atomic<unsigned long long> opted{0};
    if (bytes > 48 * 1024) {
        const cudaError_t e = opt_in_once(k, opted);
        if (e != cudaSuccess) return e;
    }
    const int tiles_x = (L.W + kTX - 1) / kTX, tiles_y = (L.H + kTY - 1) / kTY;
    k<<<tiles_x * tiles_y, kThreads, bytes, st>>>(L, Rim, L.W, L.H, g, tiles_x, disp, disp_norm);
    return cudaGetLastError();
}

template <int KIND, int R, int P, bool FILT>
cudaError_t launch_one(const ImgArg& L, const ImgArg& Rim, const VolArg& out, const Geom& g, float* fl_out,
                       cudaStream_t st) {
    const int bytes = (FILT ? Band<KIND, R>::floats_filtered(g) : Band<KIND, R>::floats(g)) * 4;
    auto k = cost_band_kernel<KIND, R, P, FILT>;
    static std::atomic<unsigned long long> opted{0};
    if (bytes > 48 * 1024) {
        const cudaError_t e = opt_in_once(k, opted);
        if (e != cudaSuccess) return e;
    }
    const int tiles_x = (out.W + kTX - 1) / kTX, tiles_y = (out.H + kTY - 1) / kTY;
    k<<<tiles_x * tiles_y, kThreads, bytes, st>>>(L, Rim, out, g, tiles_x, fl_out);
    return cudaGetLastError();
}

template <int KIND, bool FILT>
cudaError_t dispatch_r(int r, const ImgArg& L, const ImgArg& Rim, const VolArg& out, const Geom& g, float* fl_out,
                       cudaStream_t st) {
    switch (r) {
        case 1: return launch_one<KIND, 1, 16, FILT>(L, Rim, out, g, fl_out, st);
        case 2: return launch_one<KIND, 2, 16, FILT>(L, Rim, out, g, fl_out, st);
        case 3: return launch_one<KIND, 3, 16, FILT>(L, Rim, out, g, fl_out, st);
        default: return launch_one<KIND, 4, 16, FILT>(L, Rim, out, g, fl_out, st);
    }
}

long long band_floats(int kind, int r, int D, bool filt) {
    const long long lbw = left_band_width(r), rbw = kTX + D - 1 + 2 * r;
    long long f;
    if (kind == TDV_COST_BT) {
        f = 3LL * kTX * kTY + 3LL * kTY * (kTX + D - 1);
        if (filt) {
            const long long w = kTX + D + 1, rows = kTY + 4;
            f += (long long)kTY * (kTX + 2) + (long long)kTY * w + rows * (w + 4) + rows * w;
        }
        return f;
    }
    f = (long long)(kTY + 2 * r) * (lbw + rbw);
    if (kind == TDV_COST_NCC) f += (long long)kTX * kTY + (long long)kTY * (kTX + D - 1);
    if (filt) {
        const long long w = lbw > rbw ? lbw : rbw, rows = kTY + 2 * r + 4;
        f += rows * (w + 4) + rows * w;
    }
    return f;
}

}  // namespace

bool cost_banded_supported(int kind, int radius, int D, bool prefiltered) {
    if (kind != TDV_COST_BT && (radius < 1 || radius > 4)) return false;
    return band_floats(kind, kind == TDV_COST_BT ? 0 : radius, D, prefiltered) * 4 <= kMaxBandBytes;
}

cudaError_t launch_fast_wta_banded(const ImgArg& L, const ImgArg& R, int D, int radius, uint16_t* disp,
                                  float* disp_norm, cudaStream_t st) {
    Geom g;
    g.D = D;
    g.Dw = D >= 32 ? 32 : D > 8 ? 16 : 8;
    g.G = 32 / g.Dw;
    g.lbw = left_band_width(radius);
    g.rbw = kTX + D - 1 + 2 * radius;
    switch (radius) {
        case 1: return launch_fastwta_r<1>(L, R, g, disp, disp_norm, st);
        case 2: return launch_fastwta_r<2>(L, R, g, disp, disp_norm, st);
        case 3: return launch_fastwta_r<3>(L, R, g, disp, disp_norm, st);
        default: return launch_fastwta_r<4>(L, R, g, disp, disp_norm, st);
    }
}

cudaError_t launch_cost_banded(const ImgArg& L, const ImgArg& R, int kind, int radius, const VolArg& out,
                               bool prefiltered, float* left_filtered, cudaStream_t st) {
    Geom g;
    g.D = out.D;
    g.Dw = out.D >= 32 ? 32 : out.D > 8 ? 16 : 8;
    g.G = 32 / g.Dw;
    const int r = kind == TDV_COST_BT ? 0 : radius;
    g.lbw = left_band_width(r);
    g.rbw = kTX + out.D - 1 + 2 * r;
    if (prefiltered) {
        if (kind == TDV_COST_BT) return launch_one<TDV_COST_BT, 0, 8, true>(L, R, out, g, left_filtered, st);
        if (kind == TDV_COST_SSD) return dispatch_r<TDV_COST_SSD, true>(radius, L, R, out, g, left_filtered, st);
        return dispatch_r<TDV_COST_NCC, true>(radius, L, R, out, g, left_filtered, st);
    }
    if (kind == TDV_COST_BT) return launch_one<TDV_COST_BT, 0, 8, false>(L, R, out, g, nullptr, st);
    if (kind == TDV_COST_SSD) return dispatch_r<TDV_COST_SSD, false>(radius, L, R, out, g, nullptr, st);
    return dispatch_r<TDV_COST_NCC, false>(radius, L, R, out, g, nullptr, st);
}

}  // namespace tdv
