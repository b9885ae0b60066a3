// Image stages either side of the matching path, one thread per output
// pixel, tiles staged in shared memory where a window is read:
//   grey conversion (tdvision/misc.cpp:29-32), rectification remap
//   (rectificationcv.cpp:298-310), pre-filters (medianfiltercpu.cpp:15,
//   medianfilter.cu:37-57), the disparity opening (dilate.cpp:18-19), a 3x3
//   median, sub-pixel refinement and reprojection to 3D
//   (glreprojection.cpp:30-55, directreprojector.hpp:17-20,
//   cvreprojector.cpp:45-60).
// Float expressions use explicit round-to-nearest intrinsics in a fixed
// order, so each result equals the oracle's restatement bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "gauss5.cuh"
#include "tdv_internal.hpp"

namespace tdv {

namespace {

constexpr int kTX = 32, kTY = 8;  // output tile of a block

// ---------------------------------------------------------------- grey
// 1/255 scale of each 8-bit value: cvConvertScale computes it in double and
// rounds to float, which for all 256 values equals the correctly rounded
// float quotient v / 255.
__device__ __forceinline__ float scale255(uint8_t v) { return __fdiv_rn((float)v, 255.0f); }

__global__ void to_gray_kernel(RasterArg c, float* gray) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= c.W) return;
    const uint8_t* p = (const uint8_t*)c.ptr + (size_t)y * c.pitch + (size_t)x * 3;
    const float r = scale255(p[0]), g = scale255(p[1]), b = scale255(p[2]);
    gray[(size_t)y * c.W + x] =
        __fadd_rn(__fadd_rn(__fmul_rn(r, 0.299f), __fmul_rn(g, 0.587f)), __fmul_rn(b, 0.114f));
}

// ---------------------------------------------------------------- remap
// Bilinear sample at a position rounded to 1/32 pixel (cvRound of 32x the
// map value, round to nearest even); taps outside the source read 0.
template <typename T, int C>
__global__ void remap_kernel(RasterArg src, const float* __restrict__ mx, const float* __restrict__ my,
                             RasterArg dst) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= dst.W) return;
    const size_t m = (size_t)y * dst.W + x;
    // saturate far-away coordinates (every tap then lies outside)
    const float fxs = fminf(fmaxf(__fmul_rn(mx[m], 32.0f), -1.0e9f), 1.0e9f);
    const float fys = fminf(fmaxf(__fmul_rn(my[m], 32.0f), -1.0e9f), 1.0e9f);
    const int X = __float2int_rn(fxs), Y = __float2int_rn(fys);
    const int ix = X >> 5, iy = Y >> 5, fx = X & 31, fy = Y & 31;
    T* out = (T*)((char*)dst.ptr + (size_t)y * dst.pitch) + (size_t)x * C;
    const bool in00 = ix >= 0 && ix < src.W && iy >= 0 && iy < src.H;
    const bool in01 = ix + 1 >= 0 && ix + 1 < src.W && iy >= 0 && iy < src.H;
    const bool in10 = ix >= 0 && ix < src.W && iy + 1 >= 0 && iy + 1 < src.H;
    const bool in11 = ix + 1 >= 0 && ix + 1 < src.W && iy + 1 >= 0 && iy + 1 < src.H;
    auto tap = [&](int xx, int yy, int c, bool in) -> T {
        return in ? ((const T*)((const char*)src.ptr + (size_t)yy * src.pitch))[(size_t)xx * C + c] : (T)0;
    };
    if (sizeof(T) == 1) {
        // weights (1-ay)(1-ax), (1-ay)ax, ay(1-ax), ay ax in units of 2^-15
        const int w00 = (32 - fy) * (32 - fx) * 32, w01 = (32 - fy) * fx * 32;
        const int w10 = fy * (32 - fx) * 32, w11 = fy * fx * 32;
#pragma unroll
        for (int c = 0; c < C; c++) {
            const int acc = (int)tap(ix, iy, c, in00) * w00 + (int)tap(ix + 1, iy, c, in01) * w01 +
                            (int)tap(ix, iy + 1, c, in10) * w10 + (int)tap(ix + 1, iy + 1, c, in11) * w11;
            out[c] = (T)min(255, max(0, (acc + (1 << 14)) >> 15));
        }
    } else {
        const float ax = (float)fx * 0.03125f, ay = (float)fy * 0.03125f;
        const float w00 = __fmul_rn(__fsub_rn(1.0f, ay), __fsub_rn(1.0f, ax));
        const float w01 = __fmul_rn(__fsub_rn(1.0f, ay), ax);
        const float w10 = __fmul_rn(ay, __fsub_rn(1.0f, ax));
        const float w11 = __fmul_rn(ay, ax);
#pragma unroll
        for (int c = 0; c < C; c++) {
            float s = __fmul_rn((float)tap(ix, iy, c, in00), w00);
            s = __fadd_rn(s, __fmul_rn((float)tap(ix + 1, iy, c, in01), w01));
            s = __fadd_rn(s, __fmul_rn((float)tap(ix, iy + 1, c, in10), w10));
            s = __fadd_rn(s, __fmul_rn((float)tap(ix + 1, iy + 1, c, in11), w11));
            out[c] = (T)s;
        }
    }
}

// ------------------------------------------------------ rectification maps
struct RectArg {
    double ir[9];                       // inv(P[:, :3] R), row-major
    double fx, fy, cx, cy;
    double k1, k2, p1, p2, k3, k4, k5, k6;
};

__global__ void rectify_maps_kernel(RectArg a, int W, int H, float* mapx, float* mapy) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= W) return;
    const double dj = j, di = i;
    auto lin = [&](int r) {
        return __dadd_rn(__dadd_rn(__dmul_rn(dj, a.ir[3 * r]), __dmul_rn(di, a.ir[3 * r + 1])), a.ir[3 * r + 2]);
    };
    const double w = __ddiv_rn(1.0, lin(2));
    const double x = __dmul_rn(lin(0), w), y = __dmul_rn(lin(1), w);
    const double x2 = __dmul_rn(x, x), y2 = __dmul_rn(y, y);
    const double r2 = __dadd_rn(x2, y2);
    const double xy2 = __dmul_rn(__dmul_rn(2.0, x), y);
    auto poly = [&](double c3, double c2, double c1) {  // 1 + ((c3 r2 + c2) r2 + c1) r2
        return __dadd_rn(1.0, __dmul_rn(__dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(c3, r2), c2), r2), c1), r2));
    };
    const double kr = __ddiv_rn(poly(a.k3, a.k2, a.k1), poly(a.k6, a.k5, a.k4));
    const double u = __dadd_rn(
        __dmul_rn(a.fx, __dadd_rn(__dadd_rn(__dmul_rn(x, kr), __dmul_rn(a.p1, xy2)),
                                  __dmul_rn(a.p2, __dadd_rn(r2, __dmul_rn(2.0, x2))))),
        a.cx);
    const double v = __dadd_rn(
        __dmul_rn(a.fy, __dadd_rn(__dadd_rn(__dmul_rn(y, kr), __dmul_rn(a.p1, __dadd_rn(r2, __dmul_rn(2.0, y2)))),
                                  __dmul_rn(a.p2, xy2))),
        a.cy);
    mapx[(size_t)i * W + j] = __double2float_rn(u);
    mapy[(size_t)i * W + j] = __double2float_rn(v);
}

// ---------------------------------------------------------------- tiles
__device__ __forceinline__ float img_clamped(const ImgArg& im, int x, int y) {
    x = min(max(x, 0), im.W - 1);
    y = min(max(y, 0), im.H - 1);
    const size_t o = (size_t)y * im.pitch + x;
    if (im.u8) return __fmul_rn((float)((const uint8_t*)im.ptr)[o], im.scale);
    return __fmul_rn(((const float*)im.ptr)[o], im.scale);
}


// 5x5 Gaussian, replicated borders: input tile (kTY+4) x (kTX+4), rows
// filtered into (kTY+4) x kTX, then columns.
__global__ void gauss5_kernel(ImgArg in, float* out) {
    __shared__ float t[kTY + 4][kTX + 4];
    __shared__ float r[kTY + 4][kTX];
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    const int tid = threadIdx.y * kTX + threadIdx.x;
    for (int i = tid; i < (kTY + 4) * (kTX + 4); i += kTX * kTY) {
        const int ty = i / (kTX + 4), tx = i % (kTX + 4);
        t[ty][tx] = img_clamped(in, x0 + tx - 2, y0 + ty - 2);
    }
    __syncthreads();
    for (int i = tid; i < (kTY + 4) * kTX; i += kTX * kTY) {
        const int ty = i / kTX, tx = i % kTX;
        r[ty][tx] = gauss5(t[ty][tx], t[ty][tx + 1], t[ty][tx + 2], t[ty][tx + 3], t[ty][tx + 4]);
    }
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y, x = x0 + tx, y = y0 + ty;
    if (x < in.W && y < in.H)
        out[(size_t)y * in.W + x] = gauss5(r[ty][tx], r[ty + 1][tx], r[ty + 2][tx], r[ty + 3][tx], r[ty + 4][tx]);
}

// Median of N values (N odd) by forgetful selection: a buffer of N/2 + 2
// values; each step moves the buffer's minimum to its front and maximum to
// its back, drops the minimum and overwrites the maximum with the next input
// (neither can be the median).  Every index is a compile-time constant.
template <int N, typename T, typename Get>
__device__ __forceinline__ T forgetful_median(Get&& get) {
    constexpr int B = N / 2 + 2;
    T v[B];
#pragma unroll
    for (int i = 0; i < B; i++) v[i] = get(i);
    auto cswap = [](T& a, T& b) {
        const T lo = a < b ? a : b, hi = a < b ? b : a;
        a = lo;
        b = hi;
    };
#pragma unroll
    for (int step = 0; step < N - B; step++) {
        const int lo = step;
        cswap(v[lo], v[B - 1]);
#pragma unroll
        for (int j = lo + 1; j < B - 1; j++) {
            cswap(v[lo], v[j]);
            cswap(v[j], v[B - 1]);
        }
        v[B - 1] = get(B + step);
    }
    // three values left: v[N-B .. B-1]
    constexpr int L = N - B;
    cswap(v[L], v[L + 1]);
    cswap(v[L + 1], v[L + 2]);
    cswap(v[L], v[L + 1]);
    return v[L + 1];
}

// 7x7 median, replicated borders.
__global__ void median7_kernel(ImgArg in, float* out) {
    __shared__ float t[kTY + 6][kTX + 6];
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    const int tid = threadIdx.y * kTX + threadIdx.x;
    for (int i = tid; i < (kTY + 6) * (kTX + 6); i += kTX * kTY) {
        const int ty = i / (kTX + 6), tx = i % (kTX + 6);
        t[ty][tx] = img_clamped(in, x0 + tx - 3, y0 + ty - 3);
    }
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y, x = x0 + tx, y = y0 + ty;
    if (x >= in.W || y >= in.H) return;
    out[(size_t)y * in.W + x] = forgetful_median<49, float>([&](int i) { return t[ty + i / 7][tx + i % 7]; });
}

// --------------------------------------------------------- disparity maps
template <typename T>
__device__ __forceinline__ T ld_map(const RasterArg& m, int x, int y) {
    return ((const T*)((const char*)m.ptr + (size_t)y * m.pitch))[x];
}
template <typename T>
__device__ __forceinline__ void st_map(const RasterArg& m, int x, int y, T v) {
    ((T*)((char*)m.ptr + (size_t)y * m.pitch))[x] = v;
}

// 7x7 minimum (MAX = false) or maximum over the window clipped at the
// borders (outside pixels take the neutral value), rows then columns.
template <typename T, bool MAX>
__global__ void minmax7_kernel(RasterArg in, RasterArg out, T neutral) {
    __shared__ T t[kTY + 6][kTX + 6];
    __shared__ T r[kTY + 6][kTX];
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    const int tid = threadIdx.y * kTX + threadIdx.x;
    for (int i = tid; i < (kTY + 6) * (kTX + 6); i += kTX * kTY) {
        const int ty = i / (kTX + 6), tx = i % (kTX + 6);
        const int x = x0 + tx - 3, y = y0 + ty - 3;
        t[ty][tx] = (x >= 0 && x < in.W && y >= 0 && y < in.H) ? ld_map<T>(in, x, y) : neutral;
    }
    __syncthreads();
    auto pick = [](T a, T b) { return MAX ? (a < b ? b : a) : (b < a ? b : a); };
    for (int i = tid; i < (kTY + 6) * kTX; i += kTX * kTY) {
        const int ty = i / kTX, tx = i % kTX;
        T v = t[ty][tx];
#pragma unroll
        for (int k = 1; k < 7; k++) v = pick(v, t[ty][tx + k]);
        r[ty][tx] = v;
    }
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y, x = x0 + tx, y = y0 + ty;
    if (x >= in.W || y >= in.H) return;
    T v = r[ty][tx];
#pragma unroll
    for (int k = 1; k < 7; k++) v = pick(v, r[ty + k][tx]);
    st_map<T>(out, x, y, v);
}

// 3x3 median, replicated borders.
template <typename T>
__global__ void median3_kernel(RasterArg in, RasterArg out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= in.W) return;
    const T m = forgetful_median<9, T>([&](int i) {
        const int xx = min(max(x + i % 3 - 1, 0), in.W - 1), yy = min(max(y + i / 3 - 1, 0), in.H - 1);
        return ld_map<T>(in, xx, yy);
    });
    st_map<T>(out, x, y, m);
}

// ------------------------------------------------------------- sub-pixel
__global__ void subpixel_kernel(const float* __restrict__ S, int W, int H, int D,
                                const uint16_t* __restrict__ disp, float* out) {
    const size_t n = (size_t)W * H;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int d = disp[p];
        float v;
        if (d == 0xFFFF || d >= D) {
            v = -1.0f;
        } else {
            v = (float)d;
            if (d > 0 && d < D - 1) {
                const float* s = S + p * D + d;
                const float a = s[-1], b = s[0], c = s[1];
                const float den = __fsub_rn(__fadd_rn(a, c), __fmul_rn(2.0f, b));
                if (den > 0.0f) v = __fadd_rn(v, __fdiv_rn(__fsub_rn(a, c), __fmul_rn(2.0f, den)));
            }
        }
        out[p] = v;
    }
}

// ----------------------------------------------------------- reprojection
struct ReprojArg {
    int mode;
    float zscale;
    double q[16];
};

__global__ void reproject_kernel(RasterArg disp, RasterArg color, int has_color, ReprojArg rp, float* verts,
                                 float* cols) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= disp.W) return;
    const float d = disp.dtype == 1 ? (float)ld_map<uint16_t>(disp, x, y) : ld_map<float>(disp, x, y);
    const float fx = (float)x, fy = (float)(disp.H - y);
    float vx, vy, vz;
    if (rp.mode == 0) {
        vx = fx;
        vy = fy;
        vz = __fmul_rn(d, rp.zscale);
    } else {
        const double X = fx, Y = fy, Z = d;
        auto row = [&](int i) {
            return __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(rp.q[4 * i], X), __dmul_rn(rp.q[4 * i + 1], Y)),
                                       __dmul_rn(rp.q[4 * i + 2], Z)),
                             rp.q[4 * i + 3]);
        };
        double w = row(3);
        if (fabs(w) > (double)FLT_EPSILON) {
            w = __drcp_rn(w);
            vx = (float)__dmul_rn(row(0), w);
            vy = (float)__dmul_rn(row(1), w);
            vz = (float)__dmul_rn(row(2), w);
        } else {
            vx = vy = vz = 0.0f;
        }
        vz = __fmul_rn(vz, 24.0f);
    }
    const size_t p = (size_t)y * disp.W + x;
    verts[3 * p] = vx;
    verts[3 * p + 1] = vy;
    verts[3 * p + 2] = vz;
    if (cols) {
        float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
        if (has_color) {
            const uint8_t* c = (const uint8_t*)color.ptr + (size_t)y * color.pitch + (size_t)x * 3;
            const float k = 1.0f / 255.0f;
            c0 = __fmul_rn((float)c[0], k);
            c1 = __fmul_rn((float)c[1], k);
            c2 = __fmul_rn((float)c[2], k);
        }
        cols[3 * p] = c0;
        cols[3 * p + 1] = c1;
        cols[3 * p + 2] = c2;
    }
}

dim3 tiles(int W, int H) { return dim3((W + kTX - 1) / kTX, (H + kTY - 1) / kTY); }

}  // namespace

cudaError_t launch_to_gray(const RasterArg& c, float* gray, cudaStream_t st) {
    to_gray_kernel<<<dim3((c.W + 127) / 128, c.H), 128, 0, st>>>(c, gray);
    return cudaGetLastError();
}

cudaError_t launch_rectify_maps(const double* K, const double* dist, const double* iR, int W, int H, float* mapx,
                               float* mapy, cudaStream_t st) {
    RectArg a;
    for (int i = 0; i < 9; i++) a.ir[i] = iR[i];
    a.fx = K[0];
    a.fy = K[4];
    a.cx = K[2];
    a.cy = K[5];
    a.k1 = dist[0];
    a.k2 = dist[1];
    a.p1 = dist[2];
    a.p2 = dist[3];
    a.k3 = dist[4];
    a.k4 = dist[5];
    a.k5 = dist[6];
    a.k6 = dist[7];
    rectify_maps_kernel<<<dim3((W + 127) / 128, H), 128, 0, st>>>(a, W, H, mapx, mapy);
    return cudaGetLastError();
}

cudaError_t launch_remap(const RasterArg& src, const float* mx, const float* my, const RasterArg& dst,
                         cudaStream_t st) {
    const dim3 g((dst.W + 127) / 128, dst.H), b(128);
    if (src.dtype == 2 && src.ch == 1) remap_kernel<uint8_t, 1><<<g, b, 0, st>>>(src, mx, my, dst);
    else if (src.dtype == 2) remap_kernel<uint8_t, 3><<<g, b, 0, st>>>(src, mx, my, dst);
    else if (src.ch == 1) remap_kernel<float, 1><<<g, b, 0, st>>>(src, mx, my, dst);
    else remap_kernel<float, 3><<<g, b, 0, st>>>(src, mx, my, dst);
    return cudaGetLastError();
}

cudaError_t launch_prefilter(const ImgArg& in, int kind, float* out, cudaStream_t st) {
    if (kind == 0) gauss5_kernel<<<tiles(in.W, in.H), dim3(kTX, kTY), 0, st>>>(in, out);
    else median7_kernel<<<tiles(in.W, in.H), dim3(kTX, kTY), 0, st>>>(in, out);
    return cudaGetLastError();
}

cudaError_t launch_postfilter(const RasterArg& in, int kind, const RasterArg& out, void* scratch, cudaStream_t st) {
    if (kind == 0) {
        // opening: minimum into scratch (dense rows), then maximum into out
        RasterArg mid = in;
        mid.ptr = scratch;
        mid.pitch = (long long)in.W * (in.dtype == 1 ? 2 : 4);
        if (in.dtype == 1) {
            minmax7_kernel<uint16_t, false><<<tiles(in.W, in.H), dim3(kTX, kTY), 0, st>>>(in, mid, (uint16_t)0xFFFF);
            minmax7_kernel<uint16_t, true><<<tiles(in.W, in.H), dim3(kTX, kTY), 0, st>>>(mid, out, (uint16_t)0);
        } else {
            minmax7_kernel<float, false><<<tiles(in.W, in.H), dim3(kTX, kTY), 0, st>>>(in, mid, INFINITY);
            minmax7_kernel<float, true><<<tiles(in.W, in.H), dim3(kTX, kTY), 0, st>>>(mid, out, -INFINITY);
        }
    } else {
        const dim3 g((in.W + 127) / 128, in.H), b(128);
        if (in.dtype == 1) median3_kernel<uint16_t><<<g, b, 0, st>>>(in, out);
        else median3_kernel<float><<<g, b, 0, st>>>(in, out);
    }
    return cudaGetLastError();
}

cudaError_t launch_subpixel(const float* S, int W, int H, int D, const uint16_t* disp, float* out,
                            cudaStream_t st) {
    const size_t n = (size_t)W * H;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    subpixel_kernel<<<blocks, 256, 0, st>>>(S, W, H, D, disp, out);
    return cudaGetLastError();
}

cudaError_t launch_reproject(const RasterArg& disp, const RasterArg* color, int mode, float zscale,
                             const float* q, float* verts, float* cols, cudaStream_t st) {
    ReprojArg rp;
    rp.mode = mode;
    rp.zscale = zscale;
    for (int i = 0; i < 16; i++) rp.q[i] = q ? (double)q[i] : (i % 5 == 0 ? 1.0 : 0.0);
    RasterArg c{};
    if (color) c = *color;
    reproject_kernel<<<dim3((disp.W + 127) / 128, disp.H), 128, 0, st>>>(disp, c, color != nullptr, rp, verts,
                                                                        cols);
    return cudaGetLastError();
}

}  // namespace tdv
