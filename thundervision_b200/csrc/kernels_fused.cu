// Fused Birchfield-Tomasi + SGM + WTA (+ left-right check) for integer-domain
// inputs: u8 intensities used unscaled, P1/P2 multiples of 1/2, constant P2,
// STANDARD recurrence over the FULL path table, D <= 256.
//
// Exactness.  In this domain every BT cost is a multiple of 1/2 in [0, 255]
// and every path cost L = C + min(...) - m' lies in [0, 255 + P2], so all
// quantities are small multiples of 1/2.  The kernel carries them as unsigned
// 16-bit "half-units" (2x the value), two disparities per 32-bit register.
// Integer arithmetic on these is exact, so the result is bit-identical to the
// float32 recurrence of the reference (tdvision/semiglobalcpu.cpp:104-122)
// evaluated on the same values, in any summation order.  Cells with x-d < 0
// (+INF in the reference) carry a sentinel BIG = 511 + 2*P2h that can never
// win a minimum and stays bounded: every invalid L is in [BIG, BIG + P2h] and
// every invalid S in [8*BIG, 8*(BIG + P2h)] <= 65535, above any valid S.
//
// Data flow per frame (8 paths):
//   prep : BT planes for both images (I, half-sample min, half-sample max).
//   pass : V+ V- D1+ D1- D2+ D2- H+ H-, one warp per path line; lanes own
//          consecutive disparities; d-1/d+1 neighbours by byte permutes plus
//          one shuffle each way; min over d by redux.sync.  The first pass
//          stores S, the middle ones read-modify-write it, the last (H-)
//          reads it, finishes S in registers and reduces it to the disparity
//          (and the right-view disparity for the left-right check) without
//          storing it.  S lives in HBM as [y][x][d] u16, 64*PPL d per pixel.
#include <cuda_runtime.h>

#include <cstdint>

#include "tdv_internal.hpp"

namespace tdv {

namespace {

constexpr int kWarps = 4;   // warps (= path lines) per block
constexpr int kLook = 4;    // S loads issued this many steps ahead
constexpr int kRing = 256;  // right-disparity ring per warp (>= max D)

struct __align__(16) Plane {
    uint32_t i, mn, mx, pad;
};

__device__ __forceinline__ uint32_t vmin2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t vmax2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("max.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t hi_lo(uint32_t a, uint32_t b) {
    // (hi16(a), lo16(b)) as (lo, hi) of the result
    return __byte_perm(a, b, 0x5432);
}

__device__ __forceinline__ int u8_at(const ImgArg& im, int x, int y) {
    x = min(max(x, 0), im.W - 1);
    y = min(max(y, 0), im.H - 1);
    return ((const uint8_t*)im.ptr)[(size_t)y * im.pitch + x];
}

// Per pixel, in half-units: 2I, min(2I, I+I(x-1), I+I(x+1)), max(...) with
// clamp-to-edge taps (tdvision/birchfieldcost.cu:22-32).
__device__ __forceinline__ void bt_triple(const ImgArg& im, int x, int y, uint32_t& i2,
                                          uint32_t& mn, uint32_t& mx) {
    const int v = u8_at(im, x, y);
    const int a = v + u8_at(im, x - 1, y);
    const int b = v + u8_at(im, x + 1, y);
    i2 = 2 * v;
    mn = min(2 * v, min(a, b));
    mx = max(2 * v, max(a, b));
}

__global__ void prep_kernel(ImgArg L, ImgArg R, Plane* LP, Plane* RP, int W, int H) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    uint32_t i2, mn, mx;
    bt_triple(L, x, y, i2, mn, mx);
    Plane lp;
    lp.i = i2 * 0x10001u;
    lp.mn = mn * 0x10001u;
    lp.mx = mx * 0x10001u;
    lp.pad = 0;
    LP[(size_t)y * W + x] = lp;
    // right plane at xr packs (value at xr, value at xr-1): the pair of
    // disparities (d, d+1) seen from left column x reads RP[x-d].
    uint32_t j2, jn, jx, k2, kn, kx;
    bt_triple(R, x, y, j2, jn, jx);
    bt_triple(R, max(x - 1, 0), y, k2, kn, kx);
    Plane rp;
    rp.i = j2 | (k2 << 16);
    rp.mn = jn | (kn << 16);
    rp.mx = jx | (kx << 16);
    rp.pad = 0;
    RP[(size_t)y * W + x] = rp;
}

struct FK {
    const Plane* LP;
    const Plane* RP;
    uint32_t* S;  // pairs
    int W, H, D, Dp2;  // Dp2 = u32 pairs per pixel
    uint32_t P1P1, P2P2, BIGBIG;
    uint16_t* disp;
    float* disp_norm;
    uint16_t* disp_right;
    int lr_thr;
};

__device__ __forceinline__ void walk_geom(int i, int dx, int dy, int W, int H, int& sx, int& sy,
                                          int& len) {
    if (dy == 0) {
        sy = i;
        sx = dx > 0 ? 0 : W - 1;
        len = W;
        return;
    }
    if (dx == 0) {
        sx = i;
        sy = dy > 0 ? 0 : H - 1;
        len = H;
        return;
    }
    const int ye = dy > 0 ? 0 : H - 1;
    const int xe = dx > 0 ? 0 : W - 1;
    if (i < W) {
        sx = i;
        sy = ye;
    } else {
        sx = xe;
        sy = ye + dy * (i - W + 1);
    }
    const int nx = dx > 0 ? W - sx : sx + 1;
    const int ny = dy > 0 ? H - sy : sy + 1;
    len = min(nx, ny);
}

template <int PPL>
struct Vec;
template <>
struct Vec<1> {
    static __device__ __forceinline__ void ld(const uint32_t* p, uint32_t* v) { v[0] = __ldcs(p); }
    static __device__ __forceinline__ void st(uint32_t* p, const uint32_t* v) { __stcs(p, v[0]); }
};
template <>
struct Vec<2> {
    static __device__ __forceinline__ void ld(const uint32_t* p, uint32_t* v) {
        const uint2 t = __ldcs((const uint2*)p);
        v[0] = t.x;
        v[1] = t.y;
    }
    static __device__ __forceinline__ void st(uint32_t* p, const uint32_t* v) {
        __stcs((uint2*)p, make_uint2(v[0], v[1]));
    }
};
template <>
struct Vec<4> {
    static __device__ __forceinline__ void ld(const uint32_t* p, uint32_t* v) {
        const uint4 t = __ldcs((const uint4*)p);
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    }
    static __device__ __forceinline__ void st(uint32_t* p, const uint32_t* v) {
        __stcs((uint4*)p, make_uint4(v[0], v[1], v[2], v[3]));
    }
};

// BT costs (half-units) of this lane's disparity pairs at left pixel (x, y).
template <int PPL>
__device__ __forceinline__ void bt_pairs(const FK& k, int x, int y, int base, uint32_t* c) {
    const uint4 lp = __ldg((const uint4*)&k.LP[(size_t)y * k.W + x]);
    const Plane* rrow = k.RP + (size_t)y * k.W;
    const int lim = min(x + 1, k.D);  // valid d < lim
#pragma unroll
    for (int q = 0; q < PPL; q++) {
        const int d = base + 2 * q;
        const int xr = max(x - d, 0);
        const uint4 rp = __ldg((const uint4*)&rrow[xr]);
        // .x = I, .y = half-sample min, .z = half-sample max
        const uint32_t A = vmax2(lp.x, rp.y) - vmin2(lp.x, rp.z);
        const uint32_t B = vmax2(rp.x, lp.y) - vmin2(rp.x, lp.z);
        uint32_t v = vmin2(A, B);
        if (d + 1 >= lim) v = (d < lim) ? ((v & 0xFFFFu) | (k.BIGBIG & 0xFFFF0000u)) : k.BIGBIG;
        c[q] = v;
    }
}

template <int PPL>
__device__ __forceinline__ uint32_t warp_min_pairs(const uint32_t* L) {
    uint32_t t = L[0];
#pragma unroll
    for (int q = 1; q < PPL; q++) t = vmin2(t, L[q]);
    t = min(t & 0xFFFFu, t >> 16);
    return __reduce_min_sync(0xFFFFFFFFu, t);
}

// MODE 0: first pass (store S); 1: middle pass (S += L); 2: last pass (final
// S -> WTA, optional left-right check; only launched for H-).
template <int PPL, int MODE>
__global__ void __launch_bounds__(kWarps * 32) fused_pass(FK k, int dx, int dy, int nwalks) {
    extern __shared__ uint32_t smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int walk = blockIdx.x * kWarps + warp;
    if (walk >= nwalks) return;
    int sx, sy, len;
    walk_geom(walk, dx, dy, k.W, k.H, sx, sy, len);
    const int base = lane * 2 * PPL;

    const bool lr = MODE == 2 && k.lr_thr >= 0;
    uint32_t* ring = smem + warp * kRing;
    uint16_t* rowL = (uint16_t*)(smem + kWarps * kRing) + (size_t)warp * 2 * k.W;
    uint16_t* rowR = rowL + k.W;
    if (lr) {
        for (int i = lane; i < kRing; i += 32) ring[i] = 0xFFFFFFFFu;
        __syncwarp();
    }

    uint32_t L[PPL], c[PPL], s[PPL];
    uint32_t sb[kLook][PPL];
    auto sptr = [&](int t) -> uint32_t* {
        const int x = sx + t * dx, y = sy + t * dy;
        return k.S + ((size_t)y * k.W + x) * k.Dp2 + lane * PPL;
    };
    auto finish = [&](int x, int y, const uint32_t* sv) {
        // WTA: lowest (S, d) -- ties to the lowest d (tdvision/wtacpu.cpp:26-30)
        uint32_t key = 0xFFFFFFFFu;
#pragma unroll
        for (int q = 0; q < PPL; q++) {
            const uint32_t d = base + 2 * q;
            key = min(key, ((sv[q] & 0xFFFFu) << 8) | d);
            key = min(key, ((sv[q] >> 16) << 8) | (d + 1));
            if (lr) {
                // right view: candidate for xr = x - d
                const int xr0 = x - (int)d, xr1 = xr0 - 1;
                if (xr0 >= 0) {
                    uint32_t& r0 = ring[xr0 & (kRing - 1)];
                    r0 = min(r0, ((sv[q] & 0xFFFFu) << 8) | d);
                }
                if (xr1 >= 0) {
                    uint32_t& r1 = ring[xr1 & (kRing - 1)];
                    r1 = min(r1, ((sv[q] >> 16) << 8) | (d + 1));
                }
            }
        }
        key = __reduce_min_sync(0xFFFFFFFFu, key);
        const uint16_t dl = (uint16_t)(key & 0xFFu);
        if (lr) {
            __syncwarp();
            if (lane == 0) {
                uint32_t& r = ring[x & (kRing - 1)];
                rowR[x] = (uint16_t)(r & 0xFFu);
                r = 0xFFFFFFFFu;
                rowL[x] = dl;
            }
            __syncwarp();
        } else if (lane == 0) {
            const size_t o = (size_t)y * k.W + x;
            if (k.disp) k.disp[o] = dl;
            if (k.disp_norm) k.disp_norm[o] = __fdiv_rn((float)dl, (float)k.D);
        }
    };

    // step 0: L = C at the path start
    int x = sx, y = sy;
    bt_pairs<PPL>(k, x, y, base, c);
#pragma unroll
    for (int q = 0; q < PPL; q++) L[q] = c[q];
    if (MODE == 0) {
        Vec<PPL>::st(sptr(0), L);
    } else {
        Vec<PPL>::ld(sptr(0), s);
#pragma unroll
        for (int q = 0; q < PPL; q++) s[q] += L[q];
        if (MODE == 1) Vec<PPL>::st(sptr(0), s);
        else finish(x, y, s);
    }
    uint32_t m = warp_min_pairs<PPL>(L);
    if (MODE != 0) {
#pragma unroll
        for (int u = 0; u < kLook; u++)
            if (1 + u < len) Vec<PPL>::ld(sptr(1 + u), sb[u]);
    }

    for (int t0 = 1; t0 < len; t0 += kLook) {
#pragma unroll
        for (int u = 0; u < kLook; u++) {
            const int t = t0 + u;
            if (t < len) {
                x += dx;
                y += dy;
                bt_pairs<PPL>(k, x, y, base, c);
                const uint32_t MM = m * 0x10001u;
                const uint32_t MP2 = MM + k.P2P2;
                uint32_t up = __shfl_up_sync(0xFFFFFFFFu, L[PPL - 1], 1);
                uint32_t dn = __shfl_down_sync(0xFFFFFFFFu, L[0], 1);
                if (lane == 0) up = k.BIGBIG;
                if (lane == 31) dn = k.BIGBIG;
                uint32_t Ln[PPL];
#pragma unroll
                for (int q = 0; q < PPL; q++) {
                    const uint32_t lm = hi_lo(q > 0 ? L[q - 1] : up, L[q]);
                    const uint32_t lp = hi_lo(L[q], q < PPL - 1 ? L[q + 1] : dn);
                    uint32_t tv = vmin2(lm, lp) + k.P1P1;
                    tv = vmin2(vmin2(tv, L[q]), MP2);
                    Ln[q] = tv + c[q] - MM;
                }
#pragma unroll
                for (int q = 0; q < PPL; q++) L[q] = Ln[q];
                if (MODE == 0) {
                    Vec<PPL>::st(sptr(t), L);
                } else {
#pragma unroll
                    for (int q = 0; q < PPL; q++) s[q] = sb[u][q] + L[q];
                    if (t + kLook < len) Vec<PPL>::ld(sptr(t + kLook), sb[u]);
                    if (MODE == 1) Vec<PPL>::st(sptr(t), s);
                    else finish(x, y, s);
                }
                m = warp_min_pairs<PPL>(L);
            }
        }
    }

    if (lr) {
        __syncwarp();
        const int yy = sy;
        for (int xx = lane; xx < k.W; xx += 32) {
            const int dl = rowL[xx];
            const int xr = xx - dl;
            const bool bad = xr < 0 || abs(dl - (int)rowR[xr]) > k.lr_thr;
            const size_t o = (size_t)yy * k.W + xx;
            if (k.disp) k.disp[o] = bad ? (uint16_t)0xFFFF : (uint16_t)dl;
            if (k.disp_norm) k.disp_norm[o] = bad ? -1.0f : __fdiv_rn((float)dl, (float)k.D);
            if (k.disp_right) k.disp_right[o] = rowR[xx];
        }
    }
}

int nwalks_for(int dx, int dy, int W, int H) {
    if (dy == 0) return H;
    if (dx == 0) return W;
    return W + H - 1;
}

template <int PPL>
cudaError_t run_fused(const FK& k, int paths, cudaStream_t st, Timer* tm) {
    static const char* names8[8] = {"fused_pass_V+", "fused_pass_V-", "fused_pass_D1+", "fused_pass_D1-",
                                    "fused_pass_D2+", "fused_pass_D2-", "fused_pass_H+", "fused_pass_H-_wta"};
    static const char* names4[4] = {"fused_pass_V+", "fused_pass_V-", "fused_pass_H+", "fused_pass_H-_wta"};
    static const int dirs8[8][2] = {{0, 1}, {0, -1}, {1, 1}, {-1, -1}, {-1, 1}, {1, -1}, {1, 0}, {-1, 0}};
    static const int dirs4[4][2] = {{0, 1}, {0, -1}, {1, 0}, {-1, 0}};
    const int n = paths == 4 ? 4 : 8;
    const size_t lr_smem = (size_t)kWarps * kRing * 4 + (size_t)kWarps * 2 * k.W * 2;
    for (int p = 0; p < n; p++) {
        const int dx = paths == 4 ? dirs4[p][0] : dirs8[p][0];
        const int dy = paths == 4 ? dirs4[p][1] : dirs8[p][1];
        const int nw = nwalks_for(dx, dy, k.W, k.H);
        const int blocks = (nw + kWarps - 1) / kWarps;
        if (p == 0) {
            fused_pass<PPL, 0><<<blocks, kWarps * 32, 0, st>>>(k, dx, dy, nw);
        } else if (p < n - 1) {
            fused_pass<PPL, 1><<<blocks, kWarps * 32, 0, st>>>(k, dx, dy, nw);
        } else {
            const size_t sm = k.lr_thr >= 0 ? lr_smem : 0;
            if (sm > 48 * 1024) {
                cudaError_t e = cudaFuncSetAttribute(fused_pass<PPL, 2>,
                                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                if (e != cudaSuccess) return e;
            }
            fused_pass<PPL, 2><<<blocks, kWarps * 32, sm, st>>>(k, dx, dy, nw);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (tm) tm->mark(paths == 4 ? names4[p] : names8[p]);
    }
    return cudaSuccess;
}

int ppl_for(int D) { return D <= 64 ? 1 : (D <= 128 ? 2 : 4); }

}  // namespace

size_t fused_plane_bytes(int W, int H) { return (size_t)2 * W * H * sizeof(Plane); }

size_t fused_agg_bytes(int W, int H, int D) {
    return (size_t)W * H * 64 * ppl_for(D) * sizeof(uint16_t);
}

cudaError_t launch_fused(const FusedArgs& a, cudaStream_t st, Timer* tm) {
    Plane* LP = (Plane*)a.planes;
    Plane* RP = LP + (size_t)a.W * a.H;
    dim3 pb(128), pg((a.W + 127) / 128, a.H);
    prep_kernel<<<pg, pb, 0, st>>>(a.L, a.R, LP, RP, a.W, a.H);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (tm) tm->mark("fused_prep");
    FK k;
    k.LP = LP;
    k.RP = RP;
    k.S = (uint32_t*)a.agg;
    k.W = a.W;
    k.H = a.H;
    k.D = a.D;
    const int ppl = ppl_for(a.D);
    k.Dp2 = 32 * ppl;
    const uint32_t big = 511u + 2u * (uint32_t)a.p2h;
    k.P1P1 = (uint32_t)a.p1h * 0x10001u;
    k.P2P2 = (uint32_t)a.p2h * 0x10001u;
    k.BIGBIG = big * 0x10001u;
    k.disp = a.disp;
    k.disp_norm = a.disp_norm;
    k.disp_right = a.disp_right;
    k.lr_thr = a.lr_thr;
    if (ppl == 1) return run_fused<1>(k, a.paths, st, tm);
    if (ppl == 2) return run_fused<2>(k, a.paths, st, tm);
    return run_fused<4>(k, a.paths, st, tm);
}

}  // namespace tdv
