// Differentiable soft-argmin SGM (no reference counterpart): the STANDARD
// min-plus recurrence over the FULL path table with constant P1/P2,
//   L_t(d) = C_t(d) + min(L_{t-1}(d), L_{t-1}(d-1)+P1, L_{t-1}(d+1)+P1,
//                         m_{t-1}+P2) - m_{t-1},   m = min_d L,
// S = sum over directions, p_d = softmax(-S/tau), dhat = sum_d d*p_d, and its
// adjoint.  Float or double (T).
//
// Forward (per direction, one warp per path line, lanes own NPL consecutive
// disparities) records what the adjoint needs:
//   * tape mode "codes": for every cell the 2-bit choice (0 same d, 1 from
//     d-1, 2 from d+1, 3 the P2 jump; ties in that order) and for every pixel
//     the lowest argmin of L (the m used by the next step);
//   * tape mode "checkpoint k": L at every k-th step of each path; the
//     adjoint recomputes the codes of one k-step segment at a time.
// All directions run in one launch (a block's warps take consecutive walks of
// one direction): the forward stores each direction's L into its own volume
// and the argmin kernel sums them in direction order; the adjoint stores each
// direction's dC contribution into its own volume and a sum kernel adds them
// in direction order -- the same sums, in the same order, as accumulating one
// direction after another, so results are deterministic.
// Adjoint, walking each path from its end: G_t = dS_t + carry;
// dC_t += G_t; carry_{t-1}(d) = [c_t(d)=0] G_t(d) + [c_t(d+1)=1] G_t(d+1) +
// [c_t(d-1)=2] G_t(d-1) + [d = k*_{t-1}] (sum_{c=3} G_t - sum G_t);
// dP1 += sum_{c in 1,2} G_t, dP2 += sum_{c=3} G_t.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <cstdint>

#include "tdv_internal.hpp"

namespace tdv {

namespace {

constexpr uint32_t FULLM = 0xFFFFFFFFu;

template <typename T>
__device__ __forceinline__ T inf_v();
template <>
__device__ __forceinline__ float inf_v<float>() { return CUDART_INF_F; }
template <>
__device__ __forceinline__ double inf_v<double>() { return CUDART_INF; }

template <typename T>
__device__ __forceinline__ T shfl_xor(T v, int m) { return __shfl_xor_sync(FULLM, v, m); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v += shfl_xor(v, s);
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_minv(T v) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v = fmin(v, shfl_xor(v, s));
    return v;
}

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

// choice codes of one lane: 2 bits per disparity, NPL <= 16
template <int NPL>
struct CodeWord {
    static constexpr int kBytes = (NPL + 3) / 4;  // per lane per pixel
};

template <typename T, int NPL>
struct Lane {
    T v[NPL];
};

template <typename T>
struct SoftK {
    const T* C;   // HWD cost
    T* part;      // [dir][pixel][D]: per-direction L (forward) or dC contribution (backward)
    T* dS;        // HWD dLoss/dS (backward)
    uint8_t* codes;   // [dir][pixel][32 lanes][kBytes]
    uint16_t* kstar;  // [dir][pixel]
    T* ckpt;          // [dir][sum over walks of ceil(len/k)][D]
    const long long* ckpt_off;  // [dir][walk] first checkpoint index of the walk
    int W, H, D, ck;
    T p1, p2;
    T* dpen;     // [2] dP1, dP2
    T* dpen_part;  // [dir][walk][2] per-walk partial sums (summed in a fixed order)
};

__constant__ int kSoftDx[8] = {1, -1, 0, 0, 1, -1, -1, 1};
__constant__ int kSoftDy[8] = {0, 0, 1, -1, 1, -1, 1, -1};

__device__ __forceinline__ int nwalks_dev(int dx, int dy, int W, int H) {
    return dy == 0 ? H : (dx == 0 ? W : W + H - 1);
}

// This block's direction and walk-block (4 walks per block, directions in
// order); false past the last direction.
__device__ __forceinline__ bool block_dir(int nd, int W, int H, int& dir, int& wblk) {
    int b = blockIdx.x;
    for (int d = 0; d < nd; d++) {
        const int nb = (nwalks_dev(kSoftDx[d], kSoftDy[d], W, H) + 3) / 4;
        if (b < nb) {
            dir = d;
            wblk = b;
            return true;
        }
        b -= nb;
    }
    return false;
}

// L_t from L_{t-1}: returns the choice code of each disparity.
template <typename T, int NPL>
__device__ __forceinline__ void soft_step(const T* L, T m, const T* c, T p1, T p2, int lane, int d0, int D,
                                          T* Ln, uint32_t& codes) {
    const T inf = inf_v<T>();
    T up = __shfl_up_sync(FULLM, L[NPL - 1], 1);
    T dn = __shfl_down_sync(FULLM, L[0], 1);
    if (lane == 0) up = inf;
    if (lane == 31) dn = inf;
    const T mp2 = m + p2;
    codes = 0;
#pragma unroll
    for (int j = 0; j < NPL; j++) {
        const T a = L[j];
        const T b = (j > 0 ? L[j - 1] : up) + p1;
        const T e = (j < NPL - 1 ? L[j + 1] : dn) + p1;
        const T mn = fmin(a, fmin(b, fmin(e, mp2)));
        const uint32_t code = a == mn ? 0u : (b == mn ? 1u : (e == mn ? 2u : 3u));
        codes |= code << (2 * j);
        Ln[j] = (d0 + j < D) ? (c[j] + mn) - m : inf;
    }
}

// lowest-index minimum of a warp's values
template <typename T, int NPL>
__device__ __forceinline__ void warp_argmin(const T* L, int d0, T& m, int& k) {
    T lm = L[0];
#pragma unroll
    for (int j = 1; j < NPL; j++) lm = fmin(lm, L[j]);
    m = warp_minv(lm);
    int kk = 0x7FFFFFFF;
#pragma unroll
    for (int j = NPL - 1; j >= 0; j--)
        if (L[j] == m) kk = d0 + j;
    k = (int)__reduce_min_sync(FULLM, (uint32_t)kk);
}

template <typename T, int NPL>
__device__ __forceinline__ void store_codes(uint8_t* dst, uint32_t codes) {
    constexpr int B = CodeWord<NPL>::kBytes;
    if (B == 1) dst[0] = (uint8_t)codes;
    else if (B == 2) *(uint16_t*)dst = (uint16_t)codes;
    else *(uint32_t*)dst = codes;
}
template <typename T, int NPL>
__device__ __forceinline__ uint32_t load_codes(const uint8_t* src) {
    constexpr int B = CodeWord<NPL>::kBytes;
    if (B == 1) return src[0];
    if (B == 2) return *(const uint16_t*)src;
    return *(const uint32_t*)src;
}

// REC: 0 = no tape (inference), 1 = codes, 2 = checkpoints.
template <typename T, int NPL, int REC>
__global__ void __launch_bounds__(128) soft_fwd_pass(SoftK<T> k, int nd) {
    const int lane = threadIdx.x & 31;
    int dir, wblk;
    if (!block_dir(nd, k.W, k.H, dir, wblk)) return;
    const int dx = kSoftDx[dir], dy = kSoftDy[dir];
    const int nwalks = nwalks_dev(dx, dy, k.W, k.H);
    const int w = wblk * 4 + (threadIdx.x >> 5);
    if (w >= nwalks) return;
    int sx, sy, len;
    walk_geom(w, dx, dy, k.W, k.H, sx, sy, len);
    const int D = k.D;
    const int d0 = lane * NPL;
    const T inf = inf_v<T>();
    const size_t npix = (size_t)k.W * k.H;
    constexpr int CB = CodeWord<NPL>::kBytes;
    uint8_t* codes = k.codes ? k.codes + (size_t)dir * npix * 32 * CB : nullptr;
    uint16_t* kst = k.kstar ? k.kstar + (size_t)dir * npix : nullptr;
    T* ck = (REC == 2) ? k.ckpt + (size_t)k.ckpt_off[(size_t)dir * (k.W + k.H) + w] * D : nullptr;
    T* Lout = k.part + (size_t)dir * npix * D;

    T L[NPL], c[NPL], Ln[NPL];
    int x = sx, y = sy;
    size_t p = (size_t)y * k.W + x;
#pragma unroll
    for (int j = 0; j < NPL; j++) {
        const int d = d0 + j;
        c[j] = d < D ? k.C[p * D + d] : inf;
        L[j] = c[j];
        if (d < D) Lout[p * D + d] = L[j];
        if (REC == 2 && d < D) ck[d] = L[j];
    }
    T m;
    int ks;
    warp_argmin<T, NPL>(L, d0, m, ks);
    if (REC == 1 && lane == 0) kst[p] = (uint16_t)ks;
    for (int t = 1; t < len; t++) {
        x += dx;
        y += dy;
        p = (size_t)y * k.W + x;
#pragma unroll
        for (int j = 0; j < NPL; j++) {
            const int d = d0 + j;
            c[j] = d < D ? k.C[p * D + d] : inf;
        }
        uint32_t cw;
        soft_step<T, NPL>(L, m, c, k.p1, k.p2, lane, d0, D, Ln, cw);
#pragma unroll
        for (int j = 0; j < NPL; j++) {
            const int d = d0 + j;
            L[j] = Ln[j];
            if (d < D) Lout[p * D + d] = L[j];
        }
        if (REC == 1) store_codes<T, NPL>(codes + (p * 32 + lane) * CB, cw);
        if (REC == 2 && t % k.ck == 0) {
            T* dst = ck + (size_t)(t / k.ck) * D;
#pragma unroll
            for (int j = 0; j < NPL; j++)
                if (d0 + j < D) dst[d0 + j] = L[j];
        }
        warp_argmin<T, NPL>(L, d0, m, ks);
        if (REC == 1 && lane == 0) kst[p] = (uint16_t)ks;
    }
}

// S = sum of the directions' L in direction order, then the soft-argmin per
// pixel (warp per pixel): stats = (Smin, 1/Z, dhat); S stored when S_out.
template <typename T>
__global__ void soft_argmin_kernel(const T* part, int nd, int npix, int D, T tau, T* dhat, T* stats,
                                   T* S_out) {
    const int lane = threadIdx.x & 31;
    const size_t vol = (size_t)npix * D;
    constexpr int KMAXD = 8;  // D <= 256: at most 8 disparities per lane
    for (size_t p = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < (size_t)npix;
         p += ((size_t)gridDim.x * blockDim.x) >> 5) {
        T sv[KMAXD];
        T mn = inf_v<T>();
#pragma unroll
        for (int i = 0; i < KMAXD; i++) {
            const int d = lane + 32 * i;
            if (d < D) {
                T acc = part[p * D + d];
                for (int r = 1; r < nd; r++) acc = acc + part[r * vol + p * D + d];
                sv[i] = acc;
                if (S_out) S_out[p * D + d] = acc;
                mn = fmin(mn, acc);
            }
        }
        mn = warp_minv(mn);
        T z = 0, num = 0;
#pragma unroll
        for (int i = 0; i < KMAXD; i++) {
            const int d = lane + 32 * i;
            if (d < D) {
                const T e = exp(-(sv[i] - mn) / tau);
                z += e;
                num += (T)d * e;
            }
        }
        z = warp_sum(z);
        num = warp_sum(num);
        if (lane == 0) {
            const T dh = num / z;
            if (dhat) dhat[p] = dh;
            if (stats) {
                stats[3 * p] = mn;
                stats[3 * p + 1] = (T)1 / z;
                stats[3 * p + 2] = dh;
            }
        }
    }
}

// dS = g * (-1/tau) * p_d * (d - dhat)
template <typename T>
__global__ void soft_ds_kernel(const T* S, const T* stats, const T* g, int npix, int D, T tau, T* dS) {
    const size_t n = (size_t)npix * D;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t p = i / D;
        const int d = (int)(i % D);
        const T mn = stats[3 * p], zi = stats[3 * p + 1], dh = stats[3 * p + 2];
        const T pd = exp(-(S[i] - mn) / tau) * zi;
        dS[i] = g[p] * (-(T)1 / tau) * pd * ((T)d - dh);
    }
}

// Backward through one direction.  Codes and k* of the steps come from the
// tape (CK = false) or are recomputed per k-step segment from the stored
// checkpoints into shared memory (CK = true, k <= 32).
template <typename T, int NPL, bool CK>
__global__ void __launch_bounds__(128) soft_bwd_pass(SoftK<T> k, int nd) {
    constexpr int WARPS = 4;
    constexpr int KMAX = 32;
    __shared__ uint16_t sk[WARPS][KMAX + 1];
    __shared__ uint32_t segc[WARPS][KMAX][32];  // CK: codes of the segment's steps, per lane
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int dir, wblk;
    if (!block_dir(nd, k.W, k.H, dir, wblk)) return;
    const int dx = kSoftDx[dir], dy = kSoftDy[dir];
    const int nwalks = nwalks_dev(dx, dy, k.W, k.H);
    const int w = wblk * 4 + warp;
    if (w >= nwalks) return;
    int sx, sy, len;
    walk_geom(w, dx, dy, k.W, k.H, sx, sy, len);
    const int D = k.D;
    const int d0 = lane * NPL;
    const T inf = inf_v<T>();
    const size_t npix = (size_t)k.W * k.H;
    constexpr int CB = CodeWord<NPL>::kBytes;
    T* dCout = k.part + (size_t)dir * npix * D;
    const uint8_t* codes = CK ? nullptr : k.codes + (size_t)dir * npix * 32 * CB;
    const uint16_t* kst = CK ? nullptr : k.kstar + (size_t)dir * npix;
    const T* ckp = CK ? k.ckpt + (size_t)k.ckpt_off[(size_t)dir * (k.W + k.H) + w] * D : nullptr;

    T carry[NPL];
#pragma unroll
    for (int j = 0; j < NPL; j++) carry[j] = 0;
    T gp1 = 0, gp2 = 0;

    int seg_lo = 0;  // CK: steps (seg_lo, seg_hi] have codes in segc / sk
    int t = len - 1;
    while (true) {
        const int x = sx + t * dx, y = sy + t * dy;
        const size_t p = (size_t)y * k.W + x;
        T G[NPL];
#pragma unroll
        for (int j = 0; j < NPL; j++) {
            const int d = d0 + j;
            G[j] = d < D ? k.dS[p * D + d] + carry[j] : (T)0;
            if (d < D) dCout[p * D + d] = G[j];
        }
        if (t == 0) break;
        uint32_t cw;
        int ks;
        if (CK) {
            if (t <= seg_lo || t == len - 1) {
                // recompute the segment containing step t: from the checkpoint
                // at s*k, steps s*k+1 .. min(s*k+k, len-1)
                const int s0 = ((t - 1) / k.ck) * k.ck;
                const int s1 = min(s0 + k.ck, len - 1);
                T L[NPL], c[NPL], Ln[NPL];
                const T* cl = ckp + (size_t)(s0 / k.ck) * D;
#pragma unroll
                for (int j = 0; j < NPL; j++) L[j] = (d0 + j < D) ? cl[d0 + j] : inf;
                T m;
                int kk;
                warp_argmin<T, NPL>(L, d0, m, kk);
                if (lane == 0) sk[warp][0] = (uint16_t)kk;
#pragma unroll 1
                for (int u = s0 + 1; u <= s1; u++) {
                    const int xu = sx + u * dx, yu = sy + u * dy;
                    const size_t pu = (size_t)yu * k.W + xu;
#pragma unroll
                    for (int j = 0; j < NPL; j++) c[j] = (d0 + j < D) ? k.C[pu * D + d0 + j] : inf;
                    uint32_t cwu;
                    soft_step<T, NPL>(L, m, c, k.p1, k.p2, lane, d0, D, Ln, cwu);
#pragma unroll
                    for (int j = 0; j < NPL; j++) L[j] = Ln[j];
                    segc[warp][u - s0 - 1][lane] = cwu;
                    warp_argmin<T, NPL>(L, d0, m, kk);
                    if (lane == 0 && u - s0 < KMAX + 1) sk[warp][u - s0] = (uint16_t)kk;
                }
                __syncwarp();
                seg_lo = s0;
            }
            cw = segc[warp][t - seg_lo - 1][lane];
            ks = sk[warp][t - 1 - seg_lo];
        } else {
            cw = load_codes<T, NPL>(codes + (p * 32 + lane) * CB);
            const int xp = x - dx, yp = y - dy;
            ks = kst[(size_t)yp * k.W + xp];
        }
        // neighbours' G and codes
        T gup = __shfl_up_sync(FULLM, G[NPL - 1], 1);
        T gdn = __shfl_down_sync(FULLM, G[0], 1);
        uint32_t cup = __shfl_up_sync(FULLM, cw >> (2 * (NPL - 1)), 1) & 3u;
        uint32_t cdn = __shfl_down_sync(FULLM, cw, 1) & 3u;
        if (lane == 0) {
            gup = 0;
            cup = 0;
        }
        if (lane == 31) {
            gdn = 0;
            cdn = 0;
        }
        T gs = 0, g3 = 0;
#pragma unroll
        for (int j = 0; j < NPL; j++) {
            const uint32_t cj = (cw >> (2 * j)) & 3u;
            gs += G[j];
            if (cj == 3u) g3 += G[j];
            if (cj == 1u || cj == 2u) gp1 += G[j];
        }
        gp2 += g3;
        const T gm = warp_sum(g3 - gs);
#pragma unroll
        for (int j = 0; j < NPL; j++) {
            const uint32_t cj = (cw >> (2 * j)) & 3u;
            const uint32_t cplus = j < NPL - 1 ? (cw >> (2 * (j + 1))) & 3u : cdn;
            const uint32_t cminus = j > 0 ? (cw >> (2 * (j - 1))) & 3u : cup;
            const T gplus = j < NPL - 1 ? G[j + 1] : gdn;
            const T gminus = j > 0 ? G[j - 1] : gup;
            T v = 0;
            if (cj == 0u) v += G[j];
            if (cplus == 1u) v += gplus;
            if (cminus == 2u) v += gminus;
            if (d0 + j == ks) v += gm;
            carry[j] = v;
        }
        t--;
    }
    gp1 = warp_sum(gp1);
    gp2 = warp_sum(gp2);
    if (lane == 0) {
        T* part = k.dpen_part + ((size_t)dir * (k.W + k.H) + w) * 2;
        part[0] = gp1;
        part[1] = gp2;
    }
}

// dP = sum of the per-walk partials in a fixed order (deterministic).
template <typename T>
__global__ void soft_pen_reduce(const T* part, int ndir, int W, int H, T* dpen) {
    const int lane = threadIdx.x & 31;
    const int which = threadIdx.x >> 5;  // 0: P1, 1: P2
    if (which > 1) return;
    T acc = 0;
    for (int d = 0; d < ndir; d++) {
        const int dx = d == 2 || d == 3 ? 0 : 1, dy = d < 2 ? 0 : 1;
        const int nw = dy == 0 ? H : (dx == 0 ? W : W + H - 1);
        for (int w = lane; w < nw; w += 32) acc += part[((size_t)d * (W + H) + w) * 2 + which];
    }
    acc = warp_sum(acc);
    if (lane == 0) dpen[which] = acc;
}

// dC = sum of the directions' contributions in direction order.
template <typename T>
__global__ void soft_dc_sum(const T* part, int nd, size_t vol, T* dC) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < vol; i += (size_t)gridDim.x * blockDim.x) {
        T acc = part[i];
        for (int r = 1; r < nd; r++) acc = acc + part[r * vol + i];
        dC[i] = acc;
    }
}

const int kDirs8[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {-1, 1}, {1, -1}};

int nwalks_of(int dx, int dy, int W, int H) {
    if (dy == 0) return H;
    if (dx == 0) return W;
    return W + H - 1;
}

int soft_blocks(int nd, int W, int H) {
    int b = 0;
    for (int i = 0; i < nd; i++) b += (nwalks_of(kDirs8[i][0], kDirs8[i][1], W, H) + 3) / 4;
    return b;
}

template <typename T, int NPL>
cudaError_t fwd_all(SoftK<T> k, int paths, int rec, cudaStream_t st, Timer* tm) {
    const int nd = paths == 4 ? 4 : 8;
    const int blocks = soft_blocks(nd, k.W, k.H);
    if (rec == 0) soft_fwd_pass<T, NPL, 0><<<blocks, 128, 0, st>>>(k, nd);
    else if (rec == 1) soft_fwd_pass<T, NPL, 1><<<blocks, 128, 0, st>>>(k, nd);
    else soft_fwd_pass<T, NPL, 2><<<blocks, 128, 0, st>>>(k, nd);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (tm) tm->mark("soft_fwd_pass");
    return cudaSuccess;
}

template <typename T, int NPL>
cudaError_t bwd_all(SoftK<T> k, int paths, bool ck, cudaStream_t st, Timer* tm) {
    const int nd = paths == 4 ? 4 : 8;
    const int blocks = soft_blocks(nd, k.W, k.H);
    if (ck) soft_bwd_pass<T, NPL, true><<<blocks, 128, 0, st>>>(k, nd);
    else soft_bwd_pass<T, NPL, false><<<blocks, 128, 0, st>>>(k, nd);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (tm) tm->mark("soft_bwd_pass");
    return cudaSuccess;
}

int grid_for(size_t n, int block) {
    size_t g = (n + block - 1) / block;
    if (g > (size_t)148 * 32) g = (size_t)148 * 32;
    return (int)(g < 1 ? 1 : g);
}

template <typename T>
cudaError_t soft_forward_t(const SoftLaunch& L, cudaStream_t st, Timer* tm) {
    SoftK<T> k{};
    k.C = (const T*)L.cost;
    k.part = (T*)L.part;
    k.codes = (uint8_t*)L.codes;
    k.kstar = (uint16_t*)L.kstar;
    k.ckpt = (T*)L.ckpt;
    k.ckpt_off = L.ckpt_off;
    k.W = L.W;
    k.H = L.H;
    k.D = L.D;
    k.ck = L.ck;
    k.p1 = (T)L.p1;
    k.p2 = (T)L.p2;
    const int rec = L.record ? (L.ck > 0 ? 2 : 1) : 0;
    cudaError_t e;
    if (L.D <= 32) e = fwd_all<T, 1>(k, L.paths, rec, st, tm);
    else if (L.D <= 64) e = fwd_all<T, 2>(k, L.paths, rec, st, tm);
    else if (L.D <= 128) e = fwd_all<T, 4>(k, L.paths, rec, st, tm);
    else e = fwd_all<T, 8>(k, L.paths, rec, st, tm);
    if (e != cudaSuccess) return e;
    const int npix = L.W * L.H;
    soft_argmin_kernel<T><<<grid_for((size_t)npix * 32, 256), 256, 0, st>>>(
        (const T*)L.part, L.paths == 4 ? 4 : 8, npix, L.D, (T)L.tau, (T*)L.dhat, (T*)L.stats, (T*)L.S);
    if (tm) tm->mark("soft_argmin");
    return cudaGetLastError();
}

template <typename T>
cudaError_t soft_backward_t(const SoftLaunch& L, cudaStream_t st, Timer* tm) {
    SoftK<T> k{};
    k.C = (const T*)L.cost;
    k.part = (T*)L.part;
    k.dS = (T*)L.dS;
    k.codes = (uint8_t*)L.codes;
    k.kstar = (uint16_t*)L.kstar;
    k.ckpt = (T*)L.ckpt;
    k.ckpt_off = L.ckpt_off;
    k.W = L.W;
    k.H = L.H;
    k.D = L.D;
    k.ck = L.ck;
    k.p1 = (T)L.p1;
    k.p2 = (T)L.p2;
    k.dpen = (T*)L.dpen;
    k.dpen_part = (T*)L.dpen_part;
    const int npix = L.W * L.H;
    cudaError_t e;
    soft_ds_kernel<T><<<grid_for((size_t)npix * L.D, 256), 256, 0, st>>>(
        (const T*)L.S, (const T*)L.stats, (const T*)L.g, npix, L.D, (T)L.tau, (T*)L.dS);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (tm) tm->mark("soft_dS");
    const bool ck = L.ck > 0;
    if (L.D <= 32) e = bwd_all<T, 1>(k, L.paths, ck, st, tm);
    else if (L.D <= 64) e = bwd_all<T, 2>(k, L.paths, ck, st, tm);
    else if (L.D <= 128) e = bwd_all<T, 4>(k, L.paths, ck, st, tm);
    else e = bwd_all<T, 8>(k, L.paths, ck, st, tm);
    if (e != cudaSuccess) return e;
    const size_t vol = (size_t)npix * L.D;
    soft_dc_sum<T><<<grid_for(vol, 256), 256, 0, st>>>((const T*)L.part, L.paths == 4 ? 4 : 8, vol, (T*)L.dcost);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (tm) tm->mark("soft_dc_sum");
    soft_pen_reduce<T><<<1, 64, 0, st>>>(k.dpen_part, L.paths == 4 ? 4 : 8, L.W, L.H, k.dpen);
    if (tm) tm->mark("soft_pen_reduce");
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_soft_forward(const SoftLaunch& L, cudaStream_t st, Timer* tm) {
    return L.f64 ? soft_forward_t<double>(L, st, tm) : soft_forward_t<float>(L, st, tm);
}

cudaError_t launch_soft_backward(const SoftLaunch& L, cudaStream_t st, Timer* tm) {
    return L.f64 ? soft_backward_t<double>(L, st, tm) : soft_backward_t<float>(L, st, tm);
}

}  // namespace tdv
