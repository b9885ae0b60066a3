// C ABI of the image stages either side of the path (kernels_image.cu) and
// the PLY mesh writer.  Arguments are validated before any CUDA call.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "abi_common.hpp"
#include "tdv_internal.hpp"

using tdv_abi::fail;
using tdv_abi::kMaxSide;

namespace {

int dtype_bytes(int dtype) { return dtype == TDV_F32 ? 4 : (dtype == TDV_U16 ? 2 : 1); }

tdv_status check_raster(tdv_ctx* ctx, const tdv_raster* r, const char* name, bool u8_ok, bool u16_ok,
                        bool f32_ok, bool three_ok, bool one_ok) {
    if (!r) return fail(ctx, TDV_ERR_INVALID_ARG, "%s: null raster", name);
    if (!r->ptr) return fail(ctx, TDV_ERR_INVALID_ARG, "%s: null data pointer", name);
    if (r->width <= 0 || r->height <= 0 || r->width > kMaxSide || r->height > kMaxSide)
        return fail(ctx, TDV_ERR_INVALID_ARG, "%s: bad size %dx%d", name, r->width, r->height);
    const bool dt = (r->dtype == TDV_U8 && u8_ok) || (r->dtype == TDV_U16 && u16_ok) || (r->dtype == TDV_F32 && f32_ok);
    if (!dt) return fail(ctx, TDV_ERR_INVALID_ARG, "%s: unsupported dtype %d", name, r->dtype);
    if (!((r->channels == 3 && three_ok) || (r->channels == 1 && one_ok)))
        return fail(ctx, TDV_ERR_INVALID_ARG, "%s: unsupported channel count %d", name, r->channels);
    const long long row = (long long)r->width * r->channels * dtype_bytes(r->dtype);
    if (r->pitch_bytes < row)
        return fail(ctx, TDV_ERR_INVALID_ARG, "%s: pitch %d bytes < row of %lld bytes", name, r->pitch_bytes, row);
    if (r->pitch_bytes % dtype_bytes(r->dtype) != 0)
        return fail(ctx, TDV_ERR_INVALID_ARG, "%s: pitch %d not a multiple of the element size", name,
                    r->pitch_bytes);
    return TDV_OK;
}

tdv::RasterArg make_raster(const tdv_raster& r) {
    tdv::RasterArg a;
    a.ptr = r.ptr;
    a.W = r.width;
    a.H = r.height;
    a.pitch = r.pitch_bytes;
    a.dtype = r.dtype == TDV_F32 ? 0 : (r.dtype == TDV_U16 ? 1 : 2);
    a.ch = r.channels;
    return a;
}

cudaStream_t S(tdv_stream s) { return (cudaStream_t)s; }

}  // namespace

extern "C" {

tdv_status tdv_to_gray(tdv_ctx* ctx, const tdv_raster* color, float* gray, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_raster(ctx, color, "color", true, false, false, true, false));
    if (!gray) return fail(ctx, TDV_ERR_INVALID_ARG, "gray: null output");
    TDV_DEVICE_SCOPE(ctx);
    TDV_CUDA(tdv::launch_to_gray(make_raster(*color), gray, S(stream)));
    return TDV_OK;
}

tdv_status tdv_rectify_maps(tdv_ctx* ctx, const double* K, const double* dist, const double* R, const double* P,
                            int32_t width, int32_t height, float* mapx, float* mapy, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    if (!K || !dist || !R || !P || !mapx || !mapy) return fail(ctx, TDV_ERR_INVALID_ARG, "null argument");
    if (width <= 0 || height <= 0 || width > kMaxSide || height > kMaxSide)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad size %dx%d", width, height);
    for (int i = 0; i < 9; i++)
        if (!std::isfinite(K[i]) || !std::isfinite(R[i]) || !std::isfinite(P[i]))
            return fail(ctx, TDV_ERR_INVALID_ARG, "K, R and P must be finite");
    for (int i = 0; i < 8; i++)
        if (!std::isfinite(dist[i])) return fail(ctx, TDV_ERR_INVALID_ARG, "distortion must be finite");
    // M = P[:, :3] R, then its inverse by cofactors
    double M[9];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
            M[3 * r + c] = (P[3 * r] * R[c] + P[3 * r + 1] * R[3 + c]) + P[3 * r + 2] * R[6 + c];
    const double a = M[0], b = M[1], c = M[2], d = M[3], e = M[4], f = M[5], g = M[6], h = M[7], i = M[8];
    const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
    const double det = (a * A + b * B) + c * C;
    if (!(std::fabs(det) > 0.0) || !std::isfinite(det))
        return fail(ctx, TDV_ERR_INVALID_ARG, "P[:, :3] R is singular");
    const double adj[9] = {A, -(b * i - c * h), b * f - c * e, B, a * i - c * g, -(a * f - c * d),
                           C, -(a * h - b * g), a * e - b * d};
    double iR[9];
    for (int k = 0; k < 9; k++) iR[k] = adj[k] / det;
    TDV_DEVICE_SCOPE(ctx);
    TDV_CUDA(tdv::launch_rectify_maps(K, dist, iR, width, height, mapx, mapy, S(stream)));
    return TDV_OK;
}

tdv_status tdv_remap(tdv_ctx* ctx, const tdv_raster* src, const float* mapx, const float* mapy,
                     tdv_raster* dst, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_raster(ctx, src, "src", true, false, true, true, true));
    TDV_TRY(check_raster(ctx, dst, "dst", true, false, true, true, true));
    if (!mapx || !mapy) return fail(ctx, TDV_ERR_INVALID_ARG, "null map");
    if (src->dtype != dst->dtype || src->channels != dst->channels)
        return fail(ctx, TDV_ERR_INVALID_ARG, "src and dst differ in dtype or channels");
    if (src->dtype == TDV_U8 && src->channels != 3 && src->channels != 1)
        return fail(ctx, TDV_ERR_INVALID_ARG, "unsupported channel count");
    TDV_DEVICE_SCOPE(ctx);
    TDV_CUDA(tdv::launch_remap(make_raster(*src), mapx, mapy, make_raster(*dst), S(stream)));
    return TDV_OK;
}

tdv_status tdv_prefilter(tdv_ctx* ctx, const tdv_image* in, int32_t kind, float* out, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    if (!in || !in->ptr) return fail(ctx, TDV_ERR_INVALID_ARG, "in: null image");
    if (in->width <= 0 || in->height <= 0 || in->width > kMaxSide || in->height > kMaxSide || in->pitch < in->width)
        return fail(ctx, TDV_ERR_INVALID_ARG, "in: bad size or pitch");
    if (in->dtype != TDV_U8 && in->dtype != TDV_F32)
        return fail(ctx, TDV_ERR_INVALID_ARG, "in: dtype must be TDV_U8 or TDV_F32");
    if (!std::isfinite(in->scale)) return fail(ctx, TDV_ERR_INVALID_ARG, "in: scale not finite");
    if (kind != TDV_FILTER_GAUSS5 && kind != TDV_FILTER_MEDIAN7)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad filter kind %d", kind);
    if (!out) return fail(ctx, TDV_ERR_INVALID_ARG, "out: null output");
    TDV_DEVICE_SCOPE(ctx);
    TDV_CUDA(tdv::launch_prefilter(tdv::make_img(*in), kind, out, S(stream)));
    return TDV_OK;
}

tdv_status tdv_postfilter(tdv_ctx* ctx, const tdv_raster* in, int32_t kind, tdv_raster* out, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_raster(ctx, in, "in", false, true, true, false, true));
    TDV_TRY(check_raster(ctx, out, "out", false, true, true, false, true));
    if (in->dtype != out->dtype || in->width != out->width || in->height != out->height)
        return fail(ctx, TDV_ERR_INVALID_ARG, "in and out differ in size or dtype");
    if (in->ptr == out->ptr) return fail(ctx, TDV_ERR_INVALID_ARG, "in and out must not overlap");
    if (kind != TDV_POST_OPEN7 && kind != TDV_POST_MEDIAN3)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad post-filter kind %d", kind);
    TDV_DEVICE_SCOPE(ctx);
    void* scratch = nullptr;
    if (kind == TDV_POST_OPEN7) {
        TDV_TRY(tdv_abi::ensure(ctx, ctx->misc, (size_t)in->width * in->height * dtype_bytes(in->dtype)));
        scratch = ctx->misc.ptr;
    }
    TDV_CUDA(tdv::launch_postfilter(make_raster(*in), kind, make_raster(*out), scratch, S(stream)));
    return TDV_OK;
}

tdv_status tdv_subpixel(tdv_ctx* ctx, const tdv_volume* Svol, const uint16_t* disp, float* out, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    if (!Svol || !Svol->ptr) return fail(ctx, TDV_ERR_INVALID_ARG, "S: null volume");
    if (Svol->width <= 0 || Svol->height <= 0 || Svol->depth <= 0 || Svol->width > kMaxSide ||
        Svol->height > kMaxSide)
        return fail(ctx, TDV_ERR_INVALID_ARG, "S: bad size");
    if (Svol->layout != TDV_LAYOUT_HWD || Svol->dtype != TDV_F32)
        return fail(ctx, TDV_ERR_INVALID_ARG, "S: must be F32 in the HWD layout");
    if (!disp || !out) return fail(ctx, TDV_ERR_INVALID_ARG, "null disparity or output");
    TDV_DEVICE_SCOPE(ctx);
    TDV_CUDA(tdv::launch_subpixel((const float*)Svol->ptr, Svol->width, Svol->height, Svol->depth, disp, out,
                                  S(stream)));
    return TDV_OK;
}

tdv_status tdv_reproject(tdv_ctx* ctx, const tdv_raster* disp, const tdv_raster* color,
                         const tdv_reproject_params* params, float* vertices, float* colors, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_raster(ctx, disp, "disp", false, true, true, false, true));
    if (color) {
        TDV_TRY(check_raster(ctx, color, "color", true, false, false, true, false));
        if (color->width != disp->width || color->height != disp->height)
            return fail(ctx, TDV_ERR_INVALID_ARG, "color and disp differ in size");
    }
    if (!params) return fail(ctx, TDV_ERR_INVALID_ARG, "null reprojection parameters");
    if (params->mode != TDV_REPROJECT_DIRECT && params->mode != TDV_REPROJECT_Q)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad reprojection mode %d", params->mode);
    if (!std::isfinite(params->zscale)) return fail(ctx, TDV_ERR_INVALID_ARG, "zscale not finite");
    for (int i = 0; i < 16; i++)
        if (!std::isfinite(params->q[i])) return fail(ctx, TDV_ERR_INVALID_ARG, "Q has a non-finite entry");
    if (!vertices) return fail(ctx, TDV_ERR_INVALID_ARG, "null vertex output");
    TDV_DEVICE_SCOPE(ctx);
    tdv::RasterArg c{};
    if (color) c = make_raster(*color);
    TDV_CUDA(tdv::launch_reproject(make_raster(*disp), color ? &c : nullptr, params->mode, params->zscale,
                                   params->q, vertices, colors, S(stream)));
    return TDV_OK;
}

tdv_status tdv_write_ply(const char* path, const float* vertices, const float* colors, int32_t width,
                         int32_t height) {
    if (!path || !vertices || width <= 0 || height <= 0) return TDV_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, "w");
    if (!f) return TDV_ERR_INVALID_ARG;
    const long long n = (long long)width * height;
    const long long faces = (long long)(width - 1) * (height - 1);
    std::fprintf(f,
                 "ply\nformat ascii 1.0\ncomment VCGLIB generated\nelement vertex %lld\nproperty float x\n"
                 "property float y\nproperty float z\nproperty uchar red\nproperty uchar green\n"
                 "property uchar blue\nelement face %lld\nproperty list uchar int vertex_indices\n"
                 "end_header\n",
                 n, faces);
    // a float printed as an ostream prints it: 6 significant digits, %g style
    for (long long i = 0; i < n; i++) {
        int c[3] = {0, 0, 0};
        if (colors)
            for (int k = 0; k < 3; k++) c[k] = (int)(colors[3 * i + k] * 255.0f);
        std::fprintf(f, "%g %g %g %d %d %d \n", (double)vertices[3 * i], (double)vertices[3 * i + 1],
                     (double)vertices[3 * i + 2], c[0], c[1], c[2]);
    }
    for (long long row = 0; row + 1 < height; row++)
        for (long long col = 0; col + 1 < width; col++) {
            const long long a = row * width + col, b = (row + 1) * width + col;
            std::fprintf(f, "4 %lld %lld %lld %lld \n", a, b, b + 1, a + 1);
        }
    const bool ok = std::ferror(f) == 0;
    return (std::fclose(f) == 0 && ok) ? TDV_OK : TDV_ERR_INVALID_ARG;
}

}  // extern "C"
