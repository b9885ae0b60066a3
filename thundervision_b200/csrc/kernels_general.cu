// General (float32, any layout) kernels of the stage chain:
//   cost DSI writers  (BT / SSD / NCC)
//   SGM aggregation passes over a scheduled walk list (REF_CPU / REF_GPU /
//     STANDARD semantics, constant or intensity-adjusted P2)
//   WTA, left-right check, DP scanline, fused SSD+WTA.
// Float arithmetic uses explicit round-to-nearest intrinsics wherever the
// compiler could otherwise contract a multiply and an add, so each expression
// rounds exactly as the C++ oracle (built with -ffp-contract=off) does.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <cstdint>

#include "tdv_internal.hpp"

namespace tdv {

namespace {

__device__ __forceinline__ float img_at(const ImgArg& im, int x, int y) {
    x = min(max(x, 0), im.W - 1);
    y = min(max(y, 0), im.H - 1);
    const size_t o = (size_t)y * im.pitch + x;
    if (im.u8) return __fmul_rn((float)((const uint8_t*)im.ptr)[o], im.scale);
    return __fmul_rn(((const float*)im.ptr)[o], im.scale);
}

// Birchfield-Tomasi dissimilarity, tdvision/birchfieldcost.cu:14-39.
__device__ float bt_cell(const ImgArg& L, const ImgArg& R, int x, int y, int d) {
    const float lI = img_at(L, x, y);
    const float rI = img_at(R, x - d, y);
    const float laI = __fmul_rn(0.5f, __fadd_rn(lI, img_at(L, x - 1, y)));
    const float lbI = __fmul_rn(0.5f, __fadd_rn(lI, img_at(L, x + 1, y)));
    const float raI = __fmul_rn(0.5f, __fadd_rn(rI, img_at(R, x - d - 1, y)));
    const float rbI = __fmul_rn(0.5f, __fadd_rn(rI, img_at(R, x - d + 1, y)));
    const float lImi = fminf(laI, fminf(lbI, lI));
    const float lIma = fmaxf(laI, fmaxf(lbI, lI));
    const float rImi = fminf(raI, fminf(rbI, rI));
    const float rIma = fmaxf(raI, fmaxf(rbI, rI));
    const float a = fmaxf(0.0f, fmaxf(__fsub_rn(lI, rIma), __fsub_rn(rImi, lI)));
    const float b = fmaxf(0.0f, fmaxf(__fsub_rn(rI, lIma), __fsub_rn(lImi, rI)));
    return __fadd_rn(0.0f, fminf(a, b));
}

// Window SSD, rows then columns, tdvision/ssd.cu:15-29.
__device__ float ssd_cell(const ImgArg& L, const ImgArg& R, int x, int y, int d, int r) {
    float sum = 0.0f;
    for (int row = -r; row <= r; row++)
        for (int col = -r; col <= r; col++) {
            const float df = __fsub_rn(img_at(L, x + col, y + row), img_at(R, x + col - d, y + row));
            sum = __fadd_rn(sum, __fmul_rn(df, df));
        }
    return sum;
}

// Un-centred normalised cross-correlation, tdvision/crosscorrelation.cu:11-28.
__device__ float ncc_cell(const ImgArg& L, const ImgArg& R, int x, int y, int d, int r) {
    float dom = 0.0f, ls = 0.0f, rs = 0.0f;
    for (int row = -r; row <= r; row++)
        for (int col = -r; col <= r; col++) {
            const float lv = img_at(L, x + col, y + row);
            const float rv = img_at(R, x + col - d, y + row);
            dom = __fadd_rn(dom, __fmul_rn(lv, rv));
            ls = __fadd_rn(ls, __fmul_rn(lv, lv));
            rs = __fadd_rn(rs, __fmul_rn(rv, rv));
        }
    return __fsub_rn(1.0f, __fdiv_rn(dom, __fsqrt_rn(__fmul_rn(ls, rs))));
}

// Cost elements as float: a float DSI as stored; a TDV_U16 DSI holds BT of
// integer intensities in half-units (every value a multiple of 1/2, so 2v is
// an integer in [0, 510]), +INF as 0xFFFF: both directions exact.
__device__ __forceinline__ float cdec(float v) { return v; }
__device__ __forceinline__ float cdec(uint16_t u) { return u == 0xFFFFu ? CUDART_INF_F : (float)u * 0.5f; }
template <typename T>
__device__ __forceinline__ T cinf();
template <>
__device__ __forceinline__ float cinf<float>() { return CUDART_INF_F; }
template <>
__device__ __forceinline__ uint16_t cinf<uint16_t>() { return (uint16_t)0xFFFFu; }
__device__ __forceinline__ uint16_t cenc16(float v) {
    return v == CUDART_INF_F ? (uint16_t)0xFFFFu : (uint16_t)__float2uint_rn(__fmul_rn(v, 2.0f));
}

// One thread per cell in memory order (disparity fastest), so the DSI stores
// are fully coalesced whatever the layout.
__global__ void cost_kernel(ImgArg L, ImgArg R, int kind, int radius, VolArg out, int xmajor) {
    const size_t n = (size_t)out.W * out.H * out.D;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int d = (int)(i % out.D);
        const size_t p = i / out.D;
        int x, y;
        if (xmajor) { y = (int)(p % out.H); x = (int)(p / out.H); }
        else { x = (int)(p % out.W); y = (int)(p / out.W); }
        float v;
        if (kind == TDV_COST_NCC) v = (d < x + 1) ? ncc_cell(L, R, x, y, d, radius) : CUDART_INF_F;
        else if (x - d < 0) v = CUDART_INF_F;
        else if (kind == TDV_COST_BT) v = bt_cell(L, R, x, y, d);
        else v = ssd_cell(L, R, x, y, d, radius);
        if (out.u16) ((uint16_t*)out.ptr)[i] = cenc16(v);
        else ((float*)out.ptr)[i] = v;
    }
}

// Order-preserving float -> uint32 map for warp reductions with redux.sync;
// NaN maps above +INF, so a minimum ignores NaN like fminf.
__device__ __forceinline__ uint32_t ford(float f) {
    const uint32_t u = __float_as_uint(f);
    if (f != f) return 0xFFFFFFFFu;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fdeord(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }

// One warp per walk; lane l holds disparities l, l+32, ..., l+32*(NPL-1), so
// every load and store of a step moves whole 128-byte lines.  Neighbours
// d-1 and d+1 come from one rotation shuffle each: lane l-1 (or lane 31 of
// the previous group for lane 0) and lane l+1 (lane 0 of the next group for
// lane 31).  SEM and FIRST (the pass that writes S instead of adding to it)
// are compile-time, so a step carries no branch on either.
template <int NPL, int SEM, bool FIRST, typename CT>
__global__ void __launch_bounds__(128) sgm_pass_kernel(SgmArgs a, const Walk* __restrict__ walks,
                                                       int nwalks, int dx, int dy) {
    const int lane = threadIdx.x & 31;
    const int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    if (w >= nwalks) return;
    const Walk wk = walks[w];
    const int D = a.C.D;
    constexpr bool refcpu = SEM == TDV_SEM_REF_CPU;
    constexpr bool refgpu = SEM == TDV_SEM_REF_GPU;
    const int mlim = refcpu ? D - 1 : D;  // REF_CPU scans {sentinel, L(0..D-2)}
    const int src_up = (lane + 31) & 31, src_dn = (lane + 1) & 31;
    // the walk's cells: base + t * stride
    const CT* const cbase = (const CT*)a.C.ptr + wk.sx * a.C.sx + wk.sy * a.C.sy;
    float* const sbase = (float*)a.S.ptr + wk.sx * a.S.sx + wk.sy * a.S.sy;
    const long long cstride = dx * a.C.sx + dy * a.C.sy, sstride = dx * a.S.sx + dy * a.S.sy;

    float L[NPL];
    uint32_t mo = 0xFFFFFFFFu;
#pragma unroll
    for (int j = 0; j < NPL; j++) {
        const int d = lane + 32 * j;
        const float c = d < D ? cdec(cbase[d]) : CUDART_INF_F;
        if (d < mlim) mo = min(mo, ford(c));
        if (d < D) {
            if (refcpu || FIRST) {
                sbase[d] = c;
            } else if (wk.mult == 1) {
                sbase[d] = __fadd_rn(sbase[d], c);
            } else {
                a.defer[(size_t)wk.defer * D + d] = c;  // added mult times by sgm_deferred_kernel
            }
        }
        L[j] = (refgpu && d < D) ? __fadd_rn(c, a.p1) : c;
    }
    // minimum over d with fminf semantics starting from +INF: NaN ignored,
    // no candidate -> +INF
    mo = __reduce_min_sync(0xFFFFFFFFu, mo);
    float m = mo == 0xFFFFFFFFu ? CUDART_INF_F : fdeord(mo);
    const int len = wk.len;

    // P2 / |I(t) - I(t-1)| for 32 steps at a time, lane l holding step
    // t0 + l: the guide values of the next block are loaded one block ahead,
    // and a step takes its value with one shuffle.
    const bool adj = a.p2_adjust;
    auto guide_at = [&](int t) {
        return t < len ? img_at(a.guide, wk.sx + t * dx, wk.sy + t * dy) : 0.0f;
    };
    float gcur = 0.0f, gprev = 0.0f, p2blk = a.p2;
    if (adj) {
        gcur = guide_at(1 + lane);
        gprev = guide_at(lane);
    }

    // Steps 1..len-1.  The C and S loads of step t are issued K steps ahead
    // into a register ring, so a walk keeps K steps of loads in flight;
    // cells are distinct along a walk and across the walks of a pass, so a
    // prefetched S is never stale.
    constexpr int K = NPL <= 2 ? 8 : 4;
    // the ring holds the cost elements as loaded (decoded where they are
    // used, so that a 16-bit load does not have to land before the next issue)
    CT cr[K][NPL];
    float sr[K][NPL];
    auto issue = [&](int t, CT (&cs)[NPL], float (&ss)[NPL]) {
        const CT* cq = cbase + t * cstride;
        const float* sq = sbase + t * sstride;
#pragma unroll
        for (int j = 0; j < NPL; j++) {
            const int d = lane + 32 * j;
            cs[j] = d < D ? cq[d] : cinf<CT>();
            ss[j] = (!FIRST && d < D) ? sq[d] : 0.0f;
        }
    };
#pragma unroll
    for (int k = 0; k < K; k++)
        if (1 + k < len) issue(1 + k, cr[k], sr[k]);

    for (int t0 = 1; t0 < len; t0 += K) {
        if (adj && ((t0 - 1) & 31) == 0) {
            // a new block of 32 steps: its P2 values from the loaded guide
            // intensities, then the loads for the block after it
            p2blk = __fdiv_rn(a.p2, fabsf(__fsub_rn(gcur, gprev)));
            gcur = guide_at(t0 + 32 + lane);
            gprev = guide_at(t0 + 31 + lane);
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int t = t0 + k;
            if (t >= len) break;
            float* sq = sbase + t * sstride;
            const float p2a = adj ? __shfl_sync(0xFFFFFFFFu, p2blk, (t - 1) & 31) : a.p2;
            const float mp2 = __fadd_rn(m, p2a);
            float ru[NPL], rd[NPL];
#pragma unroll
            for (int j = 0; j < NPL; j++) {
                ru[j] = __shfl_sync(0xFFFFFFFFu, L[j], src_up);
                rd[j] = __shfl_sync(0xFFFFFFFFu, L[j], src_dn);
            }
            float Ln[NPL];
            uint32_t mn_o = 0xFFFFFFFFu;
#pragma unroll
            for (int j = 0; j < NPL; j++) {
                const int d = lane + 32 * j;
                const float lm = lane > 0 ? ru[j] : (j > 0 ? ru[j - 1] : CUDART_INF_F);
                const float lp = lane < 31 ? rd[j] : (j < NPL - 1 ? rd[j + 1] : CUDART_INF_F);
                const float b = __fadd_rn(lm, a.p1);
                const float e = __fadd_rn(lp, a.p1);
                float mn;
                if (refcpu) mn = smin(L[j], smin(b, smin(e, mp2)));
                else mn = fminf(L[j], fminf(b, fminf(e, mp2)));
                float v = __fsub_rn(__fadd_rn(cdec(cr[k][j]), mn), m);
                if (d >= D) v = CUDART_INF_F;
                Ln[j] = v;
                if (d < mlim) mn_o = min(mn_o, ford(v));
                if (d < D) {
                    if (FIRST) {
                        sq[d] = v;
                    } else if (wk.mult == 1) {
                        sq[d] = __fadd_rn(sr[k][j], v);
                    } else {
                        a.defer[((size_t)wk.defer + t) * D + d] = v;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < NPL; j++) L[j] = Ln[j];
            mn_o = __reduce_min_sync(0xFFFFFFFFu, mn_o);
            m = mn_o == 0xFFFFFFFFu ? CUDART_INF_F : fdeord(mn_o);
            if (t + K < len) issue(t + K, cr[k], sr[k]);
        }
    }
}

// The walks a pass repeats (the reference's table issues some walks up to
// W - H + 1 times in a row): each repeat adds the same path cost to the cell
// once more, each add rounded.  The pass kernel leaves those costs in the
// deferred buffer; here one thread per cell adds its cost mult times, so the
// repeats run in parallel over the walk's cells instead of in series along
// it.  The walks of a pass touch disjoint cells, so every cell still sees
// its updates in the reference's order.  The start cell of REF_CPU walks is
// assigned, not accumulated, by the pass kernel itself.
__global__ void sgm_deferred_kernel(SgmArgs a, const Walk* __restrict__ walks, const int32_t* __restrict__ idx,
                                    int dx, int dy, int skip_start) {
    const Walk wk = walks[idx[blockIdx.y]];
    const int D = a.S.D;
    const long long n = (long long)wk.len * D;
    float* S = (float*)a.S.ptr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int t = (int)(i / D), d = (int)(i - (long long)t * D);
        if (t == 0 && skip_start) continue;
        const int x = wk.sx + t * dx, y = wk.sy + t * dy;
        float* sp = S + x * a.S.sx + y * a.S.sy + d;
        const float v = a.defer[((size_t)wk.defer + t) * D + d];
        float acc = *sp;
        for (int q = 0; q < wk.mult; q++) acc = __fadd_rn(acc, v);
        *sp = acc;
    }
}

template <int NPL, typename CT>
cudaError_t run_passes(const SgmArgs& a, const PassSchedule& sch, cudaStream_t st, Timer* tm) {
    const int wpb = 4;
    for (size_t p = 0; p < sch.passes.size(); p++) {
        const Pass& ps = sch.passes[p];
        const int nw = (int)ps.count;
        const int blocks = (nw + wpb - 1) / wpb;
        const bool first = p == 0;
        auto kern = a.sem == TDV_SEM_REF_CPU ? (first ? sgm_pass_kernel<NPL, TDV_SEM_REF_CPU, true, CT>
                                                      : sgm_pass_kernel<NPL, TDV_SEM_REF_CPU, false, CT>)
                    : a.sem == TDV_SEM_REF_GPU ? (first ? sgm_pass_kernel<NPL, TDV_SEM_REF_GPU, true, CT>
                                                        : sgm_pass_kernel<NPL, TDV_SEM_REF_GPU, false, CT>)
                    : (first ? sgm_pass_kernel<NPL, TDV_SEM_STANDARD, true, CT>
                             : sgm_pass_kernel<NPL, TDV_SEM_STANDARD, false, CT>);
        kern<<<blocks, wpb * 32, 0, st>>>(a, sch.d_walks + ps.first, nw, ps.dx, ps.dy);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (tm) tm->mark("sgm_pass");
        if (p > 0 && ps.dcount > 0) {
            const long long cells = (long long)ps.dmaxlen * a.S.D;
            const dim3 grid((unsigned)std::min<long long>((cells + 255) / 256, 4096), (unsigned)ps.dcount);
            sgm_deferred_kernel<<<grid, 256, 0, st>>>(a, sch.d_walks, sch.d_deferred + ps.dfirst, ps.dx, ps.dy,
                                                       a.sem == TDV_SEM_REF_CPU ? 1 : 0);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
            if (tm) tm->mark("sgm_repeats");
        }
    }
    return cudaSuccess;
}

__device__ __forceinline__ void argmin_merge(uint32_t& vo, int& vd, uint32_t o2, int d2) {
    if (o2 < vo || (o2 == vo && d2 < vd)) { vo = o2; vd = d2; }
}

// Winner-take-all, one warp per pixel, strict '<' so the lowest d wins ties
// (tdvision/wtacpu.cpp:14-39); NaN never wins; no finite value -> d = 0.
template <typename T>
__global__ void wta_kernel(VolArg V, uint16_t* disp, float* disp_norm) {
    const int lane = threadIdx.x & 31;
    const size_t npix = (size_t)V.W * V.H;
    const T* base = (const T*)V.ptr;
    for (size_t p = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < npix;
         p += ((size_t)gridDim.x * blockDim.x) >> 5) {
        const int x = (int)(p % V.W), y = (int)(p / V.W);
        const T* vp = base + x * V.sx + y * V.sy;
        uint32_t bo = ford(CUDART_INF_F);
        int bd = 0x7FFFFFFF;
        for (int d = lane; d < V.D; d += 32) {
            const float v = cdec(vp[d]);
            if (v < CUDART_INF_F) argmin_merge(bo, bd, ford(v), d);
        }
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const uint32_t o2 = __shfl_xor_sync(0xFFFFFFFFu, bo, s);
            const int d2 = __shfl_xor_sync(0xFFFFFFFFu, bd, s);
            argmin_merge(bo, bd, o2, d2);
        }
        if (lane == 0) {
            const int d = bd == 0x7FFFFFFF ? 0 : bd;
            if (disp) disp[p] = (uint16_t)d;
            if (disp_norm) disp_norm[p] = __fdiv_rn((float)d, (float)V.D);
        }
    }
}

// Winner-take-all, one thread per pixel, for D a multiple of 4 and a 16-byte
// aligned volume: the pixel's D-run is read with 16-byte loads, eight in
// flight per thread, and reduced in the thread in increasing d (strict '<',
// so the lowest d wins a tie; NaN and +INF never win; no finite value ->
// d = 0), the order wta_kernel's merge gives.  Threads take pixels in memory
// order of the layout.
__global__ void __launch_bounds__(256) wta_thread_kernel(VolArg V, uint16_t* disp, float* disp_norm,
                                                         int xmajor) {
    const size_t npix = (size_t)V.W * V.H;
    const float* base = (const float*)V.ptr;
    const int n4 = V.D >> 2;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += (size_t)gridDim.x * blockDim.x) {
        int x, y;
        if (xmajor) {
            x = (int)(q / V.H);
            y = (int)(q - (size_t)x * V.H);
        } else {
            y = (int)(q / V.W);
            x = (int)(q - (size_t)y * V.W);
        }
        const float4* vp = reinterpret_cast<const float4*>(base + x * V.sx + y * V.sy);
        uint32_t bo = ford(CUDART_INF_F);
        int bd = 0x7FFFFFFF;
        for (int i0 = 0; i0 < n4; i0 += 8) {
            float4 f[8];
#pragma unroll
            for (int k = 0; k < 8; k++)
                if (i0 + k < n4) f[k] = vp[i0 + k];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                if (i0 + k >= n4) break;
                const int d = 4 * (i0 + k);
                const float v4[4] = {f[k].x, f[k].y, f[k].z, f[k].w};
#pragma unroll
                for (int e = 0; e < 4; e++)
                    if (v4[e] < CUDART_INF_F) {
                        const uint32_t o = ford(v4[e]);
                        if (o < bo) {
                            bo = o;
                            bd = d + e;
                        }
                    }
            }
        }
        const int d = bd == 0x7FFFFFFF ? 0 : bd;
        const size_t o = (size_t)y * V.W + x;
        if (disp) disp[o] = (uint16_t)d;
        if (disp_norm) disp_norm[o] = __fdiv_rn((float)d, (float)V.D);
    }
}

// Left-right check with the right-view argmin tiled through shared memory:
// one block per row; for 256 right pixels at a time and 32 disparities at a
// time the block stages S(x, y, d) for the 288 pixels those diagonals touch
// (each pixel's 32-disparity run is one 128-byte line, one warp load), in a
// 33-float row pitch so thread t reading S(xr0 + t + dd, dd) hits bank
// (t + 2 dd) mod 32.  Each thread keeps its right pixel's best (cost, d) in
// increasing d.  Then the row's left pixels are checked as in lr_kernel.
constexpr int kLrTile = 256;
template <typename T>
__global__ void __launch_bounds__(256) lr_tiled_kernel(VolArg S, uint16_t* dispL, float* disp_norm,
                                                       uint16_t* dispR, int thr) {
    extern __shared__ float lsm[];
    float* tile = lsm;                                              // [kLrTile + 32][33]
    uint16_t* sdr = reinterpret_cast<uint16_t*>(lsm + (kLrTile + 32) * 33);  // [W]
    const int y = blockIdx.x;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const T* base = (const T*)S.ptr;
    const int W = S.W, D = S.D;
    for (int xr0 = 0; xr0 < W; xr0 += kLrTile) {
        uint32_t bo = ford(CUDART_INF_F);
        int bd = 0x7FFFFFFF;
        const int xr = xr0 + t;
        for (int c = 0; c < D; c += 32) {
            __syncthreads();
            for (int i = warp; i < kLrTile + 32; i += 8) {
                const int x = xr0 + c + i, d = c + lane;
                tile[i * 33 + lane] = (x < W && d < D) ? cdec(base[x * S.sx + y * S.sy + d]) : CUDART_INF_F;
            }
            __syncthreads();
#pragma unroll 8
            for (int dd = 0; dd < 32; dd++) {
                const int d = c + dd;
                if (d < D && xr + d < W) {
                    const float v = tile[(t + dd) * 33 + dd];
                    if (v < CUDART_INF_F) {
                        const uint32_t o = ford(v);
                        if (o < bo) {
                            bo = o;
                            bd = d;
                        }
                    }
                }
            }
        }
        if (xr < W) {
            const uint16_t d = (uint16_t)(bd == 0x7FFFFFFF ? 0 : bd);
            sdr[xr] = d;
            if (dispR) dispR[(size_t)y * W + xr] = d;
        }
    }
    __syncthreads();
    for (int x = t; x < W; x += blockDim.x) {
        const size_t o = (size_t)y * W + x;
        const int dl = dispL[o];
        const int xr = x - dl;
        if (xr < 0 || abs(dl - (int)sdr[xr]) > thr) {
            dispL[o] = 0xFFFF;
            if (disp_norm) disp_norm[o] = -1.0f;
        }
    }
}

// Left-right check, one block per row.  dR(xr) = argmin_d S(xr+d, y, d) over
// xr+d < W; a left pixel is rejected (0xFFFF, d/D = -1) when x-dL < 0 or
// |dL - dR(x-dL)| > thr.
template <typename T>
__global__ void lr_kernel(VolArg S, uint16_t* dispL, float* disp_norm, uint16_t* dispR, int thr) {
    extern __shared__ uint16_t sdr[];
    const int y = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const T* base = (const T*)S.ptr;
    for (int xr = warp; xr < S.W; xr += nw) {
        uint32_t bo = ford(CUDART_INF_F);
        int bd = 0x7FFFFFFF;
        for (int d = lane; d < S.D && xr + d < S.W; d += 32) {
            const float v = cdec(base[(xr + d) * S.sx + y * S.sy + d]);
            if (v < CUDART_INF_F) argmin_merge(bo, bd, ford(v), d);
        }
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const uint32_t o2 = __shfl_xor_sync(0xFFFFFFFFu, bo, s);
            const int d2 = __shfl_xor_sync(0xFFFFFFFFu, bd, s);
            argmin_merge(bo, bd, o2, d2);
        }
        if (lane == 0) {
            const uint16_t d = (uint16_t)(bd == 0x7FFFFFFF ? 0 : bd);
            sdr[xr] = d;
            if (dispR) dispR[(size_t)y * S.W + xr] = d;
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < S.W; x += blockDim.x) {
        const size_t o = (size_t)y * S.W + x;
        const int dl = dispL[o];
        const int xr = x - dl;
        if (xr < 0 || abs(dl - (int)sdr[xr]) > thr) {
            dispL[o] = 0xFFFF;
            if (disp_norm) disp_norm[o] = -1.0f;
        }
    }
}

// DP scanline, one warp per row (tdvision/dynamicprogcpu.cpp:13-62 recurrence,
// tdvision/dynamicprog.cu:68-101 backtrack).  Choice codes (1 byte per cell,
// -1/0/+1 stored as 0/1/2) go to scratch in [y][x][d] order.  Lane l holds
// disparities l, l+32, ... (whole-line loads of C and stores of codes), the C
// columns of the next steps are in flight in a register ring, and the
// backtrack stages the codes of CW columns at a time in shared memory with
// the whole warp, so lane 0's dependent chain reads shared memory.
template <int NPL, typename T>
__global__ void __launch_bounds__(128) dp_kernel(VolArg C, uint8_t* codes, uint16_t* disp,
                                                 float* disp_norm) {
    constexpr int CW = NPL <= 8 ? 32 : 256 / NPL;  // backtrack columns per stage
    __shared__ __align__(16) uint8_t stage_all[4][CW * 32 * NPL];
    __shared__ int zs_all[4][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int y = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    if (y >= C.H) return;
    uint8_t* const stage = stage_all[wib];
    int* const zs = zs_all[wib];
    const int D = C.D, W = C.W;
    const T* base = (const T*)C.ptr;
    uint8_t* crow = codes + (size_t)y * W * D;
    const int src_up = (lane + 31) & 31, src_dn = (lane + 1) & 31;
    float A[NPL];
#pragma unroll
    for (int j = 0; j < NPL; j++) {
        const int d = lane + 32 * j;
        A[j] = d < D ? cdec(base[y * C.sy + d]) : CUDART_INF_F;
        if (d < D) crow[d] = 1;
    }
    // columns in flight: a row of D <= 64 has so little work per step that
    // 12 columns of loads ahead are needed to cover their latency (640x480
    // D=64: 0.19 -> 0.13 ms); wider rows keep their registers for the state
    constexpr int K = NPL <= 2 ? 12 : (NPL >= 16 ? 2 : 4);
    T cr[K][NPL];  // as loaded, decoded where used
    auto issue = [&](int x, T (&cs)[NPL]) {
        const T* cp = base + x * C.sx + y * C.sy;
#pragma unroll
        for (int j = 0; j < NPL; j++) {
            const int d = lane + 32 * j;
            cs[j] = d < D ? cp[d] : T(0);
        }
    };
#pragma unroll
    for (int k = 0; k < K; k++)
        if (1 + k < W) issue(1 + k, cr[k]);
    for (int x0 = 1; x0 < W; x0 += K) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int x = x0 + k;
            if (x >= W) break;
            float ru[NPL], rd[NPL];
#pragma unroll
            for (int j = 0; j < NPL; j++) {
                ru[j] = __shfl_sync(0xFFFFFFFFu, A[j], src_up);
                rd[j] = __shfl_sync(0xFFFFFFFFu, A[j], src_dn);
            }
            float An[NPL];
#pragma unroll
            for (int j = 0; j < NPL; j++) {
                const int d = lane + 32 * j;
                const float c1 = lane > 0 ? ru[j] : (j > 0 ? ru[j - 1] : CUDART_INF_F);
                const float c2 = A[j];
                const float c3 = lane < 31 ? rd[j] : (j < NPL - 1 ? rd[j + 1] : CUDART_INF_F);
                float m;
                uint8_t code;
                if (c1 < c2 && c1 < c3) { m = c1; code = 0; }
                else if (c2 < c3) { m = c2; code = 1; }
                else { m = c3; code = 2; }
                if (d < D) {
                    An[j] = __fadd_rn(cdec(cr[k][j]), m);
                    crow[(size_t)x * D + d] = code;
                } else {
                    An[j] = CUDART_INF_F;
                }
            }
#pragma unroll
            for (int j = 0; j < NPL; j++) A[j] = An[j];
            if (x + K < W) issue(x + K, cr[k]);
        }
    }
    // argmin of the last column, strict '<' from d = 0
    uint32_t bo = 0xFFFFFFFFu;
    int bd = 0x7FFFFFFF;
#pragma unroll
    for (int j = 0; j < NPL; j++) {
        const int d = lane + 32 * j;
        if (d < D) argmin_merge(bo, bd, ford(A[j]), d);
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const uint32_t o2 = __shfl_xor_sync(0xFFFFFFFFu, bo, s);
        const int d2 = __shfl_xor_sync(0xFFFFFFFFu, bd, s);
        argmin_merge(bo, bd, o2, d2);
    }
    // The reference seeds its minimum with d = 0 of the last column and only a
    // strictly smaller value replaces it, so a NaN there pins d = 0.
    const bool nan0 = __shfl_sync(0xFFFFFFFFu, A[0] != A[0] ? 1 : 0, 0) != 0;
    int z = (bd == 0x7FFFFFFF || nan0) ? 0 : bd;
    // the codes written above must be visible to the warp's staging loads
    __syncwarp();
    __threadfence_block();
    for (int xe = W - 1; xe >= 0; xe -= CW) {
        const int xs = max(0, xe - CW + 1);
        const int n = (xe - xs + 1) * D;
        const uint8_t* src = crow + (size_t)xs * D;
        if ((D & 15) == 0 && ((uintptr_t)codes & 15) == 0) {  // 16-byte aligned rows
            for (int i = lane; i < n / 16; i += 32)
                reinterpret_cast<uint4*>(stage)[i] = reinterpret_cast<const uint4*>(src)[i];
        } else {
            for (int i = lane; i < n; i += 32) stage[i] = src[i];
        }
        __syncwarp();
        if (lane == 0) {
            for (int x = xe; x >= xs; x--) {
                const int nz = z + (int)stage[(x - xs) * D + z] - 1;
                if (nz >= 0 && nz < D) z = nz;
                zs[x - xs] = z;
            }
        }
        __syncwarp();
        z = __shfl_sync(0xFFFFFFFFu, z, 0);
        if (lane <= xe - xs) {
            const int x = xs + lane;
            const size_t o = (size_t)y * W + x;
            const int zz = zs[lane];
            if (disp) disp[o] = (uint16_t)zz;
            if (disp_norm) disp_norm[o] = __fdiv_rn((float)zz, (float)D);
        }
        __syncwarp();
    }
}

// SSD window + argmin fused (tdvision/fastwta.cu:32-53), one thread per pixel.
__global__ void fast_wta_kernel(ImgArg L, ImgArg R, int D, int r, uint16_t* disp, float* disp_norm) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= L.W || y >= L.H) return;
    float best = CUDART_INF_F;
    int bd = 0;
    const int nd = min(D, x + 1);
    for (int d = 0; d < nd; d++) {
        const float v = ssd_cell(L, R, x, y, d, r);
        if (v < best) { best = v; bd = d; }
    }
    const size_t o = (size_t)y * L.W + x;
    if (disp) disp[o] = (uint16_t)bd;
    if (disp_norm) disp_norm[o] = __fdiv_rn((float)bd, (float)D);
}

int grid_for(size_t n, int block) {
    size_t g = (n + block - 1) / block;
    if (g > (size_t)148 * 64) g = (size_t)148 * 64;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace

cudaError_t launch_cost(const ImgArg& L, const ImgArg& R, int kind, int radius, const VolArg& out,
                        cudaStream_t st, Timer* tm) {
    if (cost_banded_supported(kind, radius, out.D)) {
        const cudaError_t e = launch_cost_banded(L, R, kind, radius, out, false, nullptr, st);
        if (tm) tm->mark("cost");
        return e;
    }
    // windows wider than 9x9, or bands past the shared-memory budget: one
    // thread per cell in memory order
    const size_t n = (size_t)out.W * out.H * out.D;
    const int xmajor = out.sx > out.sy ? 1 : 0;
    cost_kernel<<<grid_for(n, 256), 256, 0, st>>>(L, R, kind, radius, out, xmajor);
    if (tm) tm->mark("cost");
    return cudaGetLastError();
}

cudaError_t launch_sgm_passes(const SgmArgs& a, const PassSchedule& sch, cudaStream_t st, Timer* tm) {
    const int D = a.C.D;
    if (a.C.u16) {
        if (D <= 32) return run_passes<1, uint16_t>(a, sch, st, tm);
        if (D <= 64) return run_passes<2, uint16_t>(a, sch, st, tm);
        if (D <= 128) return run_passes<4, uint16_t>(a, sch, st, tm);
        return run_passes<8, uint16_t>(a, sch, st, tm);
    }
    if (D <= 32) return run_passes<1, float>(a, sch, st, tm);
    if (D <= 64) return run_passes<2, float>(a, sch, st, tm);
    if (D <= 128) return run_passes<4, float>(a, sch, st, tm);
    return run_passes<8, float>(a, sch, st, tm);
}

cudaError_t launch_wta(const VolArg& V, uint16_t* disp, float* disp_norm, cudaStream_t st, Timer* tm) {
    const size_t npix = (size_t)V.W * V.H;
    if (V.u16)
        wta_kernel<uint16_t><<<grid_for(npix * 32, 256), 256, 0, st>>>(V, disp, disp_norm);
    else if ((V.D & 3) == 0 && ((uintptr_t)V.ptr & 15) == 0)
        wta_thread_kernel<<<grid_for(npix, 256), 256, 0, st>>>(V, disp, disp_norm, V.sx > V.sy ? 1 : 0);
    else
        wta_kernel<float><<<grid_for(npix * 32, 256), 256, 0, st>>>(V, disp, disp_norm);
    if (tm) tm->mark("wta");
    return cudaGetLastError();
}

cudaError_t launch_lr(const VolArg& S, uint16_t* dispL, float* disp_norm, uint16_t* dispR, int thr,
                      cudaStream_t st, Timer* tm) {
    const size_t tiled = (size_t)(kLrTile + 32) * 33 * sizeof(float) + (size_t)S.W * sizeof(uint16_t);
    if (tiled <= 48 * 1024) {
        if (S.u16) lr_tiled_kernel<uint16_t><<<S.H, 256, tiled, st>>>(S, dispL, disp_norm, dispR, thr);
        else lr_tiled_kernel<float><<<S.H, 256, tiled, st>>>(S, dispL, disp_norm, dispR, thr);
    } else {
        if (S.u16) lr_kernel<uint16_t><<<S.H, 256, S.W * sizeof(uint16_t), st>>>(S, dispL, disp_norm, dispR, thr);
        else lr_kernel<float><<<S.H, 256, S.W * sizeof(uint16_t), st>>>(S, dispL, disp_norm, dispR, thr);
    }
    if (tm) tm->mark("lr_check");
    return cudaGetLastError();
}

cudaError_t launch_dp(const VolArg& C, uint16_t* disp, float* disp_norm, void* codes,
                      size_t codes_bytes, cudaStream_t st, Timer* tm) {
    (void)codes_bytes;
    const int blocks = (C.H + 3) / 4;
    const int D = C.D;
    uint8_t* cd = (uint8_t*)codes;
    if (C.u16) {
        if (D <= 32) dp_kernel<1, uint16_t><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
        else if (D <= 64) dp_kernel<2, uint16_t><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
        else if (D <= 128) dp_kernel<4, uint16_t><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
        else if (D <= 256) dp_kernel<8, uint16_t><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
        else if (D <= 512) dp_kernel<16, uint16_t><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
        else dp_kernel<32, uint16_t><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
    } else {
        if (D <= 32) dp_kernel<1, float><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
        else if (D <= 64) dp_kernel<2, float><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
        else if (D <= 128) dp_kernel<4, float><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
        else if (D <= 256) dp_kernel<8, float><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
        else if (D <= 512) dp_kernel<16, float><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
        else dp_kernel<32, float><<<blocks, 128, 0, st>>>(C, cd, disp, disp_norm);
    }
    if (tm) tm->mark("dp_scanline");
    return cudaGetLastError();
}

cudaError_t launch_fast_wta(const ImgArg& L, const ImgArg& R, int D, int radius, uint16_t* disp,
                            float* disp_norm, cudaStream_t st, Timer* tm) {
    if (cost_banded_supported(TDV_COST_SSD, radius, D)) {
        const cudaError_t e = launch_fast_wta_banded(L, R, D, radius, disp, disp_norm, st);
        if (tm) tm->mark("fast_wta");
        return e;
    }
    // radius 0 or beyond 4, or bands past the shared-memory budget
    dim3 blk(16, 16), grd((L.W + 15) / 16, (L.H + 15) / 16);
    fast_wta_kernel<<<grd, blk, 0, st>>>(L, R, D, radius, disp, disp_norm);
    if (tm) tm->mark("fast_wta");
    return cudaGetLastError();
}

}  // namespace tdv
