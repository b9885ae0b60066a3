// Host side of the C ABI: argument validation, context scratch, dispatch.
// Every entry point validates its arguments before touching CUDA, returns a
// tdv_status and records a message retrievable with tdv_last_error_string.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <new>
#include <vector>

#include "abi_common.hpp"
#include "tdv_internal.hpp"

using tdv::ImgArg;
using tdv::VolArg;

namespace {

using tdv_abi::DeviceScope;
using tdv_abi::ensure;
using tdv_abi::fail;
using tdv_abi::kMaxSide;

tdv_status check_image(tdv_ctx* ctx, const tdv_image* im, const char* name) {
    if (!im) return fail(ctx, TDV_ERR_INVALID_ARG, "%s: null image", name);
    if (!im->ptr) return fail(ctx, TDV_ERR_INVALID_ARG, "%s: null data pointer", name);
    if (im->width <= 0 || im->height <= 0 || im->width > kMaxSide || im->height > kMaxSide)
        return fail(ctx, TDV_ERR_INVALID_ARG, "%s: bad size %dx%d", name, im->width, im->height);
    if (im->pitch < im->width)
        return fail(ctx, TDV_ERR_INVALID_ARG, "%s: pitch %d < width %d", name, im->pitch, im->width);
    if (im->dtype != TDV_U8 && im->dtype != TDV_F32)
        return fail(ctx, TDV_ERR_INVALID_ARG, "%s: dtype must be TDV_U8 or TDV_F32", name);
    if (!std::isfinite(im->scale)) return fail(ctx, TDV_ERR_INVALID_ARG, "%s: scale not finite", name);
    return TDV_OK;
}

tdv_status check_volume(tdv_ctx* ctx, const tdv_volume* v, const char* name, bool allow_u16 = false) {
    if (!v) return fail(ctx, TDV_ERR_INVALID_ARG, "%s: null volume", name);
    if (!v->ptr) return fail(ctx, TDV_ERR_INVALID_ARG, "%s: null data pointer", name);
    if (v->width <= 0 || v->height <= 0 || v->depth <= 0 || v->width > kMaxSide ||
        v->height > kMaxSide)
        return fail(ctx, TDV_ERR_INVALID_ARG, "%s: bad size %dx%dx%d", name, v->width, v->height,
                    v->depth);
    if (v->layout != TDV_LAYOUT_REF_WHD && v->layout != TDV_LAYOUT_HWD)
        return fail(ctx, TDV_ERR_INVALID_ARG, "%s: bad layout %d", name, v->layout);
    if (v->dtype == TDV_U16 && allow_u16) return TDV_OK;
    if (v->dtype != TDV_F32)
        return fail(ctx, TDV_ERR_INVALID_ARG, "%s: dtype must be TDV_F32%s", name, allow_u16 ? " or TDV_U16" : "");
    return TDV_OK;
}

tdv_status check_out(tdv_ctx* ctx, const tdv_disparity* o) {
    if (!o) return fail(ctx, TDV_ERR_INVALID_ARG, "null disparity output");
    if (!o->disp && !o->disp_norm && !o->disp_right)
        return fail(ctx, TDV_ERR_INVALID_ARG, "disparity output: all pointers null");
    return TDV_OK;
}

tdv_status check_params(tdv_ctx* ctx, const tdv_sgm_params* p) {
    if (!p) return fail(ctx, TDV_ERR_INVALID_ARG, "null sgm params");
    if (!std::isfinite(p->p1) || !std::isfinite(p->p2))
        return fail(ctx, TDV_ERR_INVALID_ARG, "penalties must be finite");
    if (p->p2_mode != TDV_P2_CONST && p->p2_mode != TDV_P2_ADJUST)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad p2_mode %d", p->p2_mode);
    if (p->paths != 4 && p->paths != 8) return fail(ctx, TDV_ERR_INVALID_ARG, "paths must be 4 or 8");
    if (p->table != TDV_TABLE_FULL && p->table != TDV_TABLE_REF)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad table %d", p->table);
    if (p->semantics < TDV_SEM_STANDARD || p->semantics > TDV_SEM_REF_GPU)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad semantics %d", p->semantics);
    return TDV_OK;
}

void release_buf(tdv_ctx* ctx, tdv_ctx::Buf& b) {
    if (!b.ptr) return;
    if (ctx->release) ctx->release(b.ptr, ctx->alloc_user);
    else cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
}

cudaStream_t S(tdv_stream s) { return (cudaStream_t)s; }

// Scratch of the fused path for pairs up to W x H x D: planes and both
// aggregation volumes.
tdv_status reserve_fused(tdv_ctx* ctx, int W, int H, int D) {
    TDV_TRY(ensure(ctx, ctx->planes, tdv::fused_plane_bytes(W, H)));
    if (D <= tdv::kMaxDispSgm) {
        TDV_TRY(ensure(ctx, ctx->agg, tdv::fused_agg_bytes(W, H, D)));
        TDV_TRY(ensure(ctx, ctx->agg2, tdv::fused_agg_bytes(W, H, D)));
    }
    TDV_TRY(ensure(ctx, ctx->misc, (size_t)W * H * sizeof(uint16_t)));
    return TDV_OK;
}

// The side stream and fork/join events of the fused path's second chain.
tdv_status ensure_side(tdv_ctx* ctx) {
    if (ctx->side) return TDV_OK;
    cudaStream_t s = nullptr;
    cudaEvent_t f = nullptr, j = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&j, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (s) cudaStreamDestroy(s);
        if (f) cudaEventDestroy(f);
        return fail(ctx, TDV_ERR_CUDA, "creating the side stream failed: %s", cudaGetErrorString(e));
    }
    ctx->side = s;
    ctx->fork_ev = f;
    ctx->join_ev = j;
    return TDV_OK;
}

// The device error word is allocated (and zeroed) once per context.
tdv_status ensure_err(tdv_ctx* ctx, cudaStream_t st) {
    if (ctx->err.ptr) return TDV_OK;
    TDV_TRY(ensure(ctx, ctx->err, 16));
    TDV_CUDA(cudaMemsetAsync(ctx->err.ptr, 0, 16, st));
    return TDV_OK;
}

// The second lane of tdv_stereo_sgm_frames: its two streams and four events.
tdv_status ensure_lane(tdv_ctx* ctx) {
    if (ctx->lane_main) return TDV_OK;
    cudaStream_t m = nullptr, sd = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaError_t e = cudaStreamCreateWithFlags(&m, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sd, cudaStreamNonBlocking);
    for (int i = 0; i < 4 && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (m) cudaStreamDestroy(m);
        if (sd) cudaStreamDestroy(sd);
        for (int i = 0; i < 4; i++)
            if (ev[i]) cudaEventDestroy(ev[i]);
        return fail(ctx, TDV_ERR_CUDA, "creating the second frame lane failed: %s", cudaGetErrorString(e));
    }
    ctx->lane_main = m;
    ctx->lane_side = sd;
    ctx->lane_fork = ev[0];
    ctx->lane_join = ev[1];
    ctx->lane_start = ev[2];
    ctx->lane_done = ev[3];
    return TDV_OK;
}

tdv_status ensure_schedule(tdv_ctx* ctx, int W, int H, int table, int paths, cudaStream_t st) {
    tdv::PassSchedule& sc = ctx->sched;
    if (sc.W == W && sc.H == H && sc.table == table && sc.paths == paths && sc.d_walks) return TDV_OK;
    tdv::PassSchedule fresh;
    if (!tdv::build_schedule(W, H, table, paths, fresh))
        return fail(ctx, TDV_ERR_BAD_WORK, "path table for %dx%d has a walk outside the image", W, H);
    const size_t wbytes = (fresh.walks.size() * sizeof(tdv::Walk) + 255) & ~(size_t)255;
    TDV_TRY(ensure(ctx, ctx->sched_buf, wbytes + (fresh.deferred.size() + 1) * sizeof(int32_t)));
    sc = std::move(fresh);
    sc.d_walks = (tdv::Walk*)ctx->sched_buf.ptr;
    sc.d_deferred = (int32_t*)((char*)ctx->sched_buf.ptr + wbytes);
    TDV_CUDA(cudaMemcpyAsync(sc.d_walks, sc.walks.data(), sc.walks.size() * sizeof(tdv::Walk),
                             cudaMemcpyHostToDevice, st));
    if (!sc.deferred.empty())
        TDV_CUDA(cudaMemcpyAsync(sc.d_deferred, sc.deferred.data(), sc.deferred.size() * sizeof(int32_t),
                                 cudaMemcpyHostToDevice, st));
    // the host vector is the copy source: keep it until the copy has run
    TDV_CUDA(cudaStreamSynchronize(st));
    return TDV_OK;
}

tdv_status run_sgm(tdv_ctx* ctx, const tdv_volume* cost, const tdv_image* guide,
                   const tdv_sgm_params* p, tdv_volume* aggreg, tdv_disparity* out, cudaStream_t st) {
    const int W = cost->width, H = cost->height, D = cost->depth;
    VolArg C = tdv::make_vol(*cost);
    VolArg Sv;
    if (aggreg) {
        Sv = tdv::make_vol(*aggreg);
    } else {
        TDV_TRY(ensure(ctx, ctx->agg, (size_t)W * H * D * sizeof(float)));
        tdv_volume tmp = *cost;
        tmp.ptr = ctx->agg.ptr;
        tmp.dtype = TDV_F32;  // the aggregation is float whatever the cost's type
        Sv = tdv::make_vol(tmp);
    }
    TDV_TRY(ensure_schedule(ctx, W, H, p->table, p->paths, st));
    if (ctx->sched.defer_rows > 0)
        TDV_TRY(ensure(ctx, ctx->defer, (size_t)ctx->sched.defer_rows * D * sizeof(float)));
    tdv::SgmArgs a;
    a.defer = ctx->sched.defer_rows > 0 ? (float*)ctx->defer.ptr : nullptr;
    a.C = C;
    a.S = Sv;
    a.has_guide = guide ? 1 : 0;
    if (guide) a.guide = tdv::make_img(*guide);
    else memset(&a.guide, 0, sizeof(a.guide));
    a.p1 = p->p1;
    a.p2 = p->p2;
    a.p2_adjust = p->p2_mode == TDV_P2_ADJUST;
    a.sem = p->semantics;
    TDV_CUDA(tdv::launch_sgm_passes(a, ctx->sched, st, &ctx->timer));
    uint16_t* disp = out->disp;
    if (!disp && (out->lr_threshold >= 0 || out->disp_right)) {
        TDV_TRY(ensure(ctx, ctx->misc, (size_t)W * H * sizeof(uint16_t)));
        disp = (uint16_t*)ctx->misc.ptr;
    }
    TDV_CUDA(tdv::launch_wta(Sv, disp, out->disp_norm, st, &ctx->timer));
    if (out->lr_threshold >= 0 || out->disp_right)
        TDV_CUDA(tdv::launch_lr(Sv, disp, out->disp_norm, out->disp_right,
                                out->lr_threshold >= 0 ? out->lr_threshold : 0x7FFFFFFF, st,
                                &ctx->timer));
    return TDV_OK;
}

// ---- soft SGM tape layout -------------------------------------------------
struct SoftLayout {
    size_t S, stats, codes, kstar, off, ckpt, total;
    long long nck;
};

size_t al256(size_t v) { return (v + 255) & ~(size_t)255; }

int soft_ndir(int paths) { return paths == 4 ? 4 : 8; }

// walk lengths per direction, in the order the kernels number the walks
void soft_walk_lengths(int W, int H, int dx, int dy, std::vector<int>& out) {
    out.clear();
    if (dy == 0) {
        out.assign(H, W);
        return;
    }
    if (dx == 0) {
        out.assign(W, H);
        return;
    }
    for (int i = 0; i < W + H - 1; i++) {
        int sx, sy;
        const int ye = dy > 0 ? 0 : H - 1, xe = dx > 0 ? 0 : W - 1;
        if (i < W) {
            sx = i;
            sy = ye;
        } else {
            sx = xe;
            sy = ye + dy * (i - W + 1);
        }
        const int nx = dx > 0 ? W - sx : sx + 1;
        const int ny = dy > 0 ? H - sy : sy + 1;
        out.push_back(std::min(nx, ny));
    }
}

const int kSoftDirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {-1, 1}, {1, -1}};

SoftLayout soft_layout(int W, int H, int D, int esize, const tdv_soft_params* p,
                       std::vector<long long>* offs) {
    SoftLayout L{};
    const size_t npix = (size_t)W * H;
    const int nd = soft_ndir(p->paths);
    const int npl = D <= 32 ? 1 : (D <= 64 ? 2 : (D <= 128 ? 4 : 8));
    const int cb = (npl + 3) / 4;
    size_t o = 0;
    L.S = o;
    o = al256(o + npix * D * esize);
    L.stats = o;
    o = al256(o + npix * 3 * esize);
    if (p->checkpoint == 0) {
        L.codes = o;
        o = al256(o + (size_t)nd * npix * 32 * cb);
        L.kstar = o;
        o = al256(o + (size_t)nd * npix * 2);
    } else {
        long long n = 0;
        std::vector<int> lens;
        if (offs) offs->assign((size_t)nd * (W + H), 0);
        for (int d = 0; d < nd; d++) {
            soft_walk_lengths(W, H, kSoftDirs[d][0], kSoftDirs[d][1], lens);
            for (size_t w = 0; w < lens.size(); w++) {
                if (offs) (*offs)[(size_t)d * (W + H) + w] = n;
                n += (lens[w] + p->checkpoint - 1) / p->checkpoint;
            }
        }
        L.nck = n;
        L.off = o;
        o = al256(o + (size_t)nd * (W + H) * sizeof(long long));
        L.ckpt = o;
        o = al256(o + (size_t)n * D * esize);
    }
    L.total = o;
    return L;
}

tdv_status check_soft(tdv_ctx* ctx, const tdv_volume* cost, const tdv_soft_params* p) {
    if (!cost || !cost->ptr) return fail(ctx, TDV_ERR_INVALID_ARG, "cost: null volume");
    if (cost->width <= 0 || cost->height <= 0 || cost->depth <= 0 || cost->width > kMaxSide ||
        cost->height > kMaxSide)
        return fail(ctx, TDV_ERR_INVALID_ARG, "cost: bad size");
    if (cost->layout != TDV_LAYOUT_HWD) return fail(ctx, TDV_ERR_INVALID_ARG, "soft SGM takes the HWD layout");
    if (cost->dtype != TDV_F32 && cost->dtype != TDV_F64)
        return fail(ctx, TDV_ERR_INVALID_ARG, "soft SGM takes TDV_F32 or TDV_F64");
    if (cost->depth > tdv::kMaxDispSgm) return fail(ctx, TDV_ERR_UNSUPPORTED, "soft SGM supports D <= 256");
    if (!p) return fail(ctx, TDV_ERR_INVALID_ARG, "null soft params");
    if (p->paths != 4 && p->paths != 8) return fail(ctx, TDV_ERR_INVALID_ARG, "paths must be 4 or 8");
    if (!(p->tau > 0.0) || !std::isfinite(p->tau)) return fail(ctx, TDV_ERR_INVALID_ARG, "tau must be > 0");
    if (!std::isfinite(p->p1) || !std::isfinite(p->p2))
        return fail(ctx, TDV_ERR_INVALID_ARG, "penalties must be finite");
    if (p->checkpoint < 0 || p->checkpoint > 32)
        return fail(ctx, TDV_ERR_INVALID_ARG, "checkpoint must be in [0, 32]");
    return TDV_OK;
}

bool is_half_multiple(float v) { return v >= 0.0f && v <= 4096.0f && std::floor(2.0f * v) == 2.0f * v; }

// How an integer-domain call runs on the fused 16-bit path, if it can.
struct FusedPlan {
    bool ok = false;
    int p1h = 0, p2h = 0, off_h = 0, excl = 0, gstart = 0;
    bool weighted = false, assign = false;
};

// The fused path holds every quantity of the integer domain (u8 images used
// unscaled, constant P2, penalties multiples of 1/2) exactly in 16-bit
// half-units: the STANDARD and both reference recurrences, either table.
// Ranges (half-units, see fused_body.cuh): with the reference CPU recurrence
// path costs reach down to -OFF, OFF = 510 + max(P1h, P2h - P1h); the
// sentinel is BIG = OFF + 511 + 2 P2h and an invalid cell's sum over 8 paths,
// 8 (BIG + P2h + OFF), must fit 16 bits.
FusedPlan plan_fused(const tdv_image* left, const tdv_image* right, int D, const tdv_sgm_params* p) {
    FusedPlan f;
    if (left->dtype != TDV_U8 || right->dtype != TDV_U8 || left->scale != 1.0f || right->scale != 1.0f) return f;
    if (p->p2_mode != TDV_P2_CONST || !is_half_multiple(p->p1) || !is_half_multiple(p->p2)) return f;
    f.p1h = (int)(2.0f * p->p1);
    f.p2h = (int)(2.0f * p->p2);
    if (p->semantics == TDV_SEM_REF_GPU) f.gstart = f.p1h;
    if (p->semantics == TDV_SEM_REF_CPU) {
        if (D < 2) return f;  // its minimum over d < D-1 is then empty
        f.excl = 1;
        f.off_h = 510 + std::max(f.p1h, f.p2h - f.p1h);
        f.assign = true;
    }
    const long big = (long)f.off_h + 511 + 2L * f.p2h;
    if (8 * (big + f.p2h + f.off_h) > 65535) return f;
    f.weighted = p->table == TDV_TABLE_REF || f.assign;
    f.ok = true;
    return f;
}

// Builds (or reuses) the walk weights of the reference table / recurrence for
// a W x H pair and uploads them; false if this table's weights, or the
// 32-bit range of its repeated-line sums, fall outside the fused kernels.
bool fused_weights_ready(tdv_ctx* ctx, int W, int H, int D, const tdv_sgm_params* p, const FusedPlan& f,
                         cudaStream_t st, tdv_status* err) {
    *err = TDV_OK;
    tdv::FusedWeights& fw = ctx->fweights;
    if (fw.W != W || fw.H != H || fw.table != p->table || fw.paths != p->paths || fw.assign != (int)f.assign) {
        const char* why = nullptr;
        if (!tdv::build_fused_weights(W, H, p->table, p->paths, f.assign, fw, &why)) {
            fw = tdv::FusedWeights();
            return false;
        }
        if ((*err = ensure(ctx, ctx->fw_buf, fw.bytes)) != TDV_OK) return false;
        if (cudaMemcpyAsync(ctx->fw_buf.ptr, fw.image.data(), fw.bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            fw = tdv::FusedWeights();
            *err = fail(ctx, TDV_ERR_CUDA, "uploading the fused walk weights failed");
            return false;
        }
    }
    // a repeated line's cells add (n-1) L in 32-bit keys of (sum << 8 | d):
    // the sums must stay inside +-(2^23 - 1)
    const long maxl = (long)f.off_h + 510 + f.p2h;
    const long hi = 8 * (maxl + f.p2h) + (long)fw.max_wm1 * (maxl - f.off_h);
    const long lo = (long)fw.max_wm1 * f.off_h;
    if (hi >= (1L << 23) - 1 || lo >= (1L << 23) - 1) return false;
    if (fw.has_corner &&
        (*err = ensure(ctx, ctx->fside, (size_t)2 * H * tdv::fused_side_words(D) * sizeof(uint32_t))) != TDV_OK)
        return false;
    return true;
}

// The fused launch's arguments for one pair, without its scratch, streams
// and events (the caller's lane supplies those).
tdv::FusedArgs fused_args(tdv_ctx* ctx, const tdv_image* left, const tdv_image* right, int D,
                          const tdv_sgm_params* params, const FusedPlan& fp, const tdv_disparity* out) {
    tdv::FusedArgs a;
    a.L = tdv::make_img(*left);
    a.R = tdv::make_img(*right);
    a.W = left->width;
    a.H = left->height;
    a.D = D;
    a.p1h = fp.p1h;
    a.p2h = fp.p2h;
    a.excl = fp.excl;
    a.off_h = fp.off_h;
    a.gstart = fp.gstart;
    if (fp.weighted) {
        a.fw = &ctx->fweights;
        a.weights = (const unsigned char*)ctx->fw_buf.ptr;
    }
    a.paths = params->paths;
    a.disp = out->disp;
    a.disp_norm = out->disp_norm;
    a.disp_right = out->disp_right;
    a.lr_thr = out->lr_threshold >= 0 ? out->lr_threshold : (out->disp_right ? 0x7FFFFFFF : -1);
    a.err = (int*)ctx->err.ptr;
    return a;
}

}  // namespace

namespace tdv {

VolArg make_vol(const tdv_volume& v) {
    VolArg a;
    a.ptr = v.ptr;
    a.W = v.width;
    a.H = v.height;
    a.D = v.depth;
    a.u16 = v.dtype == TDV_U16 ? 1 : 0;
    if (v.layout == TDV_LAYOUT_REF_WHD) {
        a.sx = (long long)v.height * v.depth;
        a.sy = v.depth;
    } else {
        a.sx = v.depth;
        a.sy = (long long)v.width * v.depth;
    }
    return a;
}

ImgArg make_img(const tdv_image& im) {
    ImgArg a;
    a.ptr = im.ptr;
    a.W = im.width;
    a.H = im.height;
    a.pitch = im.pitch;
    a.u8 = im.dtype == TDV_U8 ? 1 : 0;
    a.scale = im.scale;
    return a;
}

}  // namespace tdv

extern "C" {

int32_t tdv_version(void) { return TDV_ABI_VERSION; }

const char* tdv_status_string(tdv_status s) {
    switch (s) {
        case TDV_OK: return "ok";
        case TDV_ERR_INVALID_ARG: return "invalid argument";
        case TDV_ERR_UNSUPPORTED: return "unsupported";
        case TDV_ERR_OOM: return "out of memory";
        case TDV_ERR_CUDA: return "cuda error";
        case TDV_ERR_TIMEOUT: return "timeout";
        case TDV_ERR_BAD_WORK: return "bad work item";
    }
    return "unknown status";
}

size_t tdv_volume_bytes(int32_t W, int32_t H, int32_t D, int32_t dtype) {
    if (W <= 0 || H <= 0 || D <= 0) return 0;
    size_t e = dtype == TDV_F64 ? 8 : dtype == TDV_F32 ? 4 : dtype == TDV_U16 ? 2 : 1;
    return (size_t)W * H * D * e;
}

tdv_status tdv_ctx_create(int32_t device, tdv_ctx** out) {
    if (!out) return TDV_ERR_INVALID_ARG;
    *out = nullptr;
    if (device < 0) return TDV_ERR_INVALID_ARG;
    tdv_ctx* c = new (std::nothrow) tdv_ctx;
    if (!c) return TDV_ERR_OOM;
    c->device = device;
    *out = c;
    return TDV_OK;
}

void tdv_ctx_destroy(tdv_ctx* ctx) {
    if (!ctx) return;
    const bool any = ctx->agg.ptr || ctx->cost.ptr || ctx->planes.ptr || ctx->codes.ptr ||
                     ctx->misc.ptr || ctx->sched_buf.ptr || ctx->err.ptr || ctx->soft.ptr ||
                     ctx->agg2.ptr || ctx->defer.ptr || ctx->side || ctx->fw_buf.ptr || ctx->fside.ptr ||
                     ctx->lane_main || ctx->planes_b.ptr || ctx->agg_b.ptr || ctx->agg2_b.ptr || ctx->fside_b.ptr;
    if (any) {
        DeviceScope ds(ctx->device);
        cudaDeviceSynchronize();
        release_buf(ctx, ctx->agg);
        release_buf(ctx, ctx->agg2);
        if (ctx->side) cudaStreamDestroy(ctx->side);
        if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
        if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
        release_buf(ctx, ctx->cost);
        release_buf(ctx, ctx->planes);
        release_buf(ctx, ctx->codes);
        release_buf(ctx, ctx->misc);
        release_buf(ctx, ctx->sched_buf);
        release_buf(ctx, ctx->err);
        release_buf(ctx, ctx->soft);
        release_buf(ctx, ctx->defer);
        release_buf(ctx, ctx->fw_buf);
        release_buf(ctx, ctx->fside);
        release_buf(ctx, ctx->planes_b);
        release_buf(ctx, ctx->agg_b);
        release_buf(ctx, ctx->agg2_b);
        release_buf(ctx, ctx->fside_b);
        if (ctx->lane_main) cudaStreamDestroy(ctx->lane_main);
        if (ctx->lane_side) cudaStreamDestroy(ctx->lane_side);
        for (cudaEvent_t e : {ctx->lane_fork, ctx->lane_join, ctx->lane_start, ctx->lane_done})
            if (e) cudaEventDestroy(e);
    }
    if (!ctx->timer.ev.empty()) {
        DeviceScope ds(ctx->device);
        for (cudaEvent_t e : ctx->timer.ev) cudaEventDestroy(e);
    }
    delete ctx;
}

tdv_status tdv_ctx_set_allocator(tdv_ctx* ctx, tdv_alloc_fn alloc, tdv_free_fn release, void* user) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    if ((alloc == nullptr) != (release == nullptr))
        return fail(ctx, TDV_ERR_INVALID_ARG, "allocator and release must be set together");
    if (ctx->agg.ptr || ctx->cost.ptr || ctx->planes.ptr || ctx->codes.ptr || ctx->misc.ptr ||
        ctx->sched_buf.ptr || ctx->defer.ptr)
        return fail(ctx, TDV_ERR_INVALID_ARG, "allocator must be set before any scratch exists");
    ctx->alloc = alloc;
    ctx->release = release;
    ctx->alloc_user = user;
    return TDV_OK;
}

tdv_status tdv_ctx_reserve(tdv_ctx* ctx, int32_t W, int32_t H, int32_t D) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    if (W <= 0 || H <= 0 || D <= 0 || W > kMaxSide || H > kMaxSide)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad reserve size %dx%dx%d", W, H, D);
    if (!ctx->alloc) {
        TDV_DEVICE_SCOPE(ctx);
        return reserve_fused(ctx, W, H, D);
    }
    return reserve_fused(ctx, W, H, D);
}

tdv_status tdv_ctx_enable_timing(tdv_ctx* ctx, int32_t enable) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    ctx->timer.on = enable != 0;
    ctx->timer.n = 0;
    ctx->timer.names.clear();
    ctx->timer.spans.clear();
    return TDV_OK;
}

int32_t tdv_ctx_timings(tdv_ctx* ctx, float* ms, int32_t max_entries) {
    if (!ctx || !ctx->timer.on || ctx->timer.spans.empty()) return 0;
    tdv::Timer& t = ctx->timer;
    DeviceScope ds(ctx->device);
    for (int i = 0; i < t.n; i++)
        if (cudaEventSynchronize(t.ev[i]) != cudaSuccess) return 0;
    const int n = (int)t.spans.size();
    for (int i = 0; i < n && i < max_entries && ms; i++)
        if (cudaEventElapsedTime(&ms[i], t.ev[t.spans[i].first], t.ev[t.spans[i].second]) != cudaSuccess)
            ms[i] = -1.0f;
    return n;
}

const char* tdv_ctx_timing_name(const tdv_ctx* ctx, int32_t i) {
    if (!ctx || i < 0 || i >= (int32_t)ctx->timer.names.size()) return "";
    return ctx->timer.names[i].c_str();
}

tdv_status tdv_ctx_device_status(tdv_ctx* ctx, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    if (!ctx->err.ptr) return TDV_OK;
    TDV_DEVICE_SCOPE(ctx);
    int v = 0;
    TDV_CUDA(cudaMemcpyAsync(&v, ctx->err.ptr, sizeof(int), cudaMemcpyDeviceToHost, S(stream)));
    TDV_CUDA(cudaStreamSynchronize(S(stream)));
    if (v != 0) {
        TDV_CUDA(cudaMemsetAsync(ctx->err.ptr, 0, sizeof(int), S(stream)));
        return fail(ctx, (tdv_status)v, "a kernel reported %s", tdv_status_string((tdv_status)v));
    }
    return TDV_OK;
}

size_t tdv_soft_sgm_tape_bytes(int32_t W, int32_t H, int32_t D, int32_t dtype, const tdv_soft_params* p) {
    if (W <= 0 || H <= 0 || D <= 0 || !p || (dtype != TDV_F32 && dtype != TDV_F64)) return 0;
    if (p->checkpoint < 0 || p->checkpoint > 32 || (p->paths != 4 && p->paths != 8)) return 0;
    return soft_layout(W, H, D, dtype == TDV_F64 ? 8 : 4, p, nullptr).total;
}

tdv_status tdv_soft_sgm_forward(tdv_ctx* ctx, const tdv_volume* cost, const tdv_soft_params* p, void* dhat,
                                void* tape, size_t tape_bytes, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_soft(ctx, cost, p));
    if (!dhat) return fail(ctx, TDV_ERR_INVALID_ARG, "null dhat");
    const int W = cost->width, H = cost->height, D = cost->depth;
    const int es = cost->dtype == TDV_F64 ? 8 : 4;
    SoftLayout lay = soft_layout(W, H, D, es, p, &ctx->ckpt_off_host);
    if (tape && tape_bytes < lay.total)
        return fail(ctx, TDV_ERR_INVALID_ARG, "tape of %zu bytes < %zu needed", tape_bytes, lay.total);
    TDV_DEVICE_SCOPE(ctx);
    ctx->timer.begin(S(stream));
    // scratch: one L volume per direction, then (without a tape) the statistics
    const size_t parts = (size_t)soft_ndir(p->paths) * al256((size_t)W * H * D * es);
    TDV_TRY(ensure(ctx, ctx->soft, parts + al256((size_t)W * H * 3 * es)));
    unsigned char* base = tape ? (unsigned char*)tape : nullptr;
    if (tape && p->checkpoint > 0)
        TDV_CUDA(cudaMemcpyAsync(base + lay.off, ctx->ckpt_off_host.data(),
                                 ctx->ckpt_off_host.size() * sizeof(long long), cudaMemcpyHostToDevice,
                                 S(stream)));
    tdv::SoftLaunch a{};
    a.f64 = es == 8;
    a.cost = cost->ptr;
    a.part = ctx->soft.ptr;
    a.S = tape ? base + lay.S : nullptr;
    a.stats = tape ? base + lay.stats : (unsigned char*)ctx->soft.ptr + parts;
    a.dhat = dhat;
    a.W = W;
    a.H = H;
    a.D = D;
    a.paths = p->paths;
    a.ck = tape ? p->checkpoint : 0;
    a.record = tape ? 1 : 0;
    if (tape && p->checkpoint == 0) {
        a.codes = base + lay.codes;
        a.kstar = base + lay.kstar;
    }
    if (tape && p->checkpoint > 0) {
        a.ckpt = base + lay.ckpt;
        a.ckpt_off = (const long long*)(base + lay.off);
    }
    a.p1 = p->p1;
    a.p2 = p->p2;
    a.tau = p->tau;
    TDV_CUDA(tdv::launch_soft_forward(a, S(stream), &ctx->timer));
    return TDV_OK;
}

tdv_status tdv_soft_sgm_backward(tdv_ctx* ctx, const tdv_volume* cost, const tdv_soft_params* p,
                                 const void* tape, size_t tape_bytes, const void* g_dhat, tdv_volume* dcost,
                                 void* dpen, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_soft(ctx, cost, p));
    if (!tape || !g_dhat || !dpen) return fail(ctx, TDV_ERR_INVALID_ARG, "null tape, gradient or dpen");
    if (!dcost || !dcost->ptr || dcost->width != cost->width || dcost->height != cost->height ||
        dcost->depth != cost->depth || dcost->layout != cost->layout || dcost->dtype != cost->dtype)
        return fail(ctx, TDV_ERR_INVALID_ARG, "dcost must match the cost volume");
    const int W = cost->width, H = cost->height, D = cost->depth;
    const int es = cost->dtype == TDV_F64 ? 8 : 4;
    SoftLayout lay = soft_layout(W, H, D, es, p, nullptr);
    if (tape_bytes < lay.total)
        return fail(ctx, TDV_ERR_INVALID_ARG, "tape of %zu bytes < %zu needed", tape_bytes, lay.total);
    TDV_DEVICE_SCOPE(ctx);
    ctx->timer.begin(S(stream));
    // scratch: dS, one dC contribution volume per direction, per-walk penalty sums
    const size_t ds_bytes = al256((size_t)W * H * D * es);
    const size_t parts = (size_t)soft_ndir(p->paths) * ds_bytes;
    TDV_TRY(ensure(ctx, ctx->soft, ds_bytes + parts + (size_t)8 * (W + H) * 2 * es));
    unsigned char* base = (unsigned char*)tape;
    tdv::SoftLaunch a{};
    a.f64 = es == 8;
    a.cost = cost->ptr;
    a.S = base + lay.S;
    a.stats = base + lay.stats;
    a.dS = ctx->soft.ptr;
    a.part = (unsigned char*)ctx->soft.ptr + ds_bytes;
    a.dpen_part = (unsigned char*)ctx->soft.ptr + ds_bytes + parts;
    a.dcost = dcost->ptr;
    a.g = g_dhat;
    a.dpen = dpen;
    a.W = W;
    a.H = H;
    a.D = D;
    a.paths = p->paths;
    a.ck = p->checkpoint;
    if (p->checkpoint == 0) {
        a.codes = base + lay.codes;
        a.kstar = base + lay.kstar;
    } else {
        a.ckpt = base + lay.ckpt;
        a.ckpt_off = (const long long*)(base + lay.off);
    }
    a.p1 = p->p1;
    a.p2 = p->p2;
    a.tau = p->tau;
    TDV_CUDA(tdv::launch_soft_backward(a, S(stream), &ctx->timer));
    return TDV_OK;
}

const char* tdv_last_error_string(const tdv_ctx* ctx) {
    if (!ctx) return "null context";
    return ctx->last_error.c_str();
}

tdv_status tdv_cost(tdv_ctx* ctx, const tdv_image* left, const tdv_image* right,
                    const tdv_cost_params* params, tdv_volume* out, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_image(ctx, left, "left"));
    TDV_TRY(check_image(ctx, right, "right"));
    TDV_TRY(check_volume(ctx, out, "out", true));
    if (!params) return fail(ctx, TDV_ERR_INVALID_ARG, "null cost params");
    if (params->kind < TDV_COST_BT || params->kind > TDV_COST_NCC)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad cost kind %d", params->kind);
    if (params->kind != TDV_COST_BT && (params->radius < 0 || params->radius > 15))
        return fail(ctx, TDV_ERR_INVALID_ARG, "window radius %d outside [0,15]", params->radius);
    // a 16-bit DSI holds BT of integer intensities exactly, in half-units
    if (out->dtype == TDV_U16 &&
        (params->kind != TDV_COST_BT || left->dtype != TDV_U8 || right->dtype != TDV_U8 || left->scale != 1.0f ||
         right->scale != 1.0f))
        return fail(ctx, TDV_ERR_UNSUPPORTED,
                    "a TDV_U16 DSI holds BT of TDV_U8 images at scale 1 only (half-units, exact)");
    // The reference sizes the DSI to the smaller of the two images
    // (tdvision/matchingcost.cpp:20-24).
    const int W = std::min(left->width, right->width), H = std::min(left->height, right->height);
    if (out->width != W || out->height != H)
        return fail(ctx, TDV_ERR_INVALID_ARG, "out volume %dx%d != min image size %dx%d", out->width,
                    out->height, W, H);
    TDV_DEVICE_SCOPE(ctx);
    ctx->timer.begin(S(stream));
    TDV_CUDA(tdv::launch_cost(tdv::make_img(*left), tdv::make_img(*right), params->kind,
                              params->radius, tdv::make_vol(*out), S(stream), &ctx->timer));
    return TDV_OK;
}

tdv_status tdv_cost_filtered(tdv_ctx* ctx, const tdv_image* left, const tdv_image* right,
                             const tdv_cost_params* params, int32_t filter, tdv_volume* out,
                             float* left_filtered, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_image(ctx, left, "left"));
    TDV_TRY(check_image(ctx, right, "right"));
    TDV_TRY(check_volume(ctx, out, "out"));
    if (!params) return fail(ctx, TDV_ERR_INVALID_ARG, "null cost params");
    if (params->kind < TDV_COST_BT || params->kind > TDV_COST_NCC)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad cost kind %d", params->kind);
    if (params->kind != TDV_COST_BT && (params->radius < 0 || params->radius > 15))
        return fail(ctx, TDV_ERR_INVALID_ARG, "window radius %d outside [0,15]", params->radius);
    if (filter != TDV_FILTER_GAUSS5 && filter != TDV_FILTER_MEDIAN7)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad filter kind %d", filter);
    const int W = std::min(left->width, right->width), H = std::min(left->height, right->height);
    if (out->width != W || out->height != H)
        return fail(ctx, TDV_ERR_INVALID_ARG, "out volume %dx%d != min image size %dx%d", out->width,
                    out->height, W, H);
    TDV_DEVICE_SCOPE(ctx);
    ctx->timer.begin(S(stream));
    const tdv::ImgArg L = tdv::make_img(*left), R = tdv::make_img(*right);
    const int radius = params->kind == TDV_COST_BT ? 0 : params->radius;
    if (filter == TDV_FILTER_GAUSS5 && tdv::cost_banded_supported(params->kind, radius, out->depth, true)) {
        TDV_CUDA(tdv::launch_cost_banded(L, R, params->kind, radius, tdv::make_vol(*out), true, left_filtered,
                                         S(stream)));
        ctx->timer.mark("cost_filtered");
        return TDV_OK;
    }
    // filter into scratch, then the plain cost over the filtered images
    const size_t nl = (size_t)left->width * left->height, nr = (size_t)right->width * right->height;
    TDV_TRY(ensure(ctx, ctx->misc, (nl + nr) * sizeof(float)));
    float* fl = (float*)ctx->misc.ptr;
    float* fr = fl + nl;
    TDV_CUDA(tdv::launch_prefilter(L, filter, fl, S(stream)));
    TDV_CUDA(tdv::launch_prefilter(R, filter, fr, S(stream)));
    tdv::ImgArg FL{fl, left->width, left->height, left->width, 0, 1.0f};
    tdv::ImgArg FR{fr, right->width, right->height, right->width, 0, 1.0f};
    TDV_CUDA(tdv::launch_cost(FL, FR, params->kind, params->radius, tdv::make_vol(*out), S(stream), &ctx->timer));
    if (left_filtered)
        TDV_CUDA(cudaMemcpy2DAsync(left_filtered, (size_t)W * sizeof(float), fl, (size_t)left->width * sizeof(float),
                                   (size_t)W * sizeof(float), H, cudaMemcpyDeviceToDevice, S(stream)));
    return TDV_OK;
}

tdv_status tdv_sgm(tdv_ctx* ctx, const tdv_volume* cost, const tdv_image* guide,
                   const tdv_sgm_params* params, tdv_volume* aggreg, tdv_disparity* out,
                   tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_volume(ctx, cost, "cost", true));
    TDV_TRY(check_params(ctx, params));
    TDV_TRY(check_out(ctx, out));
    if (cost->depth > tdv::kMaxDispSgm)
        return fail(ctx, TDV_ERR_UNSUPPORTED, "SGM supports D <= %d (got %d)", tdv::kMaxDispSgm,
                    cost->depth);
    if (params->p2_mode == TDV_P2_ADJUST && !guide)
        return fail(ctx, TDV_ERR_INVALID_ARG, "P2_ADJUST needs a guide image");
    if (guide) {
        TDV_TRY(check_image(ctx, guide, "guide"));
        if (guide->width < cost->width || guide->height < cost->height)
            return fail(ctx, TDV_ERR_INVALID_ARG, "guide smaller than the cost volume");
    }
    if (aggreg) {
        TDV_TRY(check_volume(ctx, aggreg, "aggreg"));
        if (aggreg->width != cost->width || aggreg->height != cost->height ||
            aggreg->depth != cost->depth || aggreg->layout != cost->layout)
            return fail(ctx, TDV_ERR_INVALID_ARG, "aggreg must match the cost volume's size and layout");
        if (aggreg->ptr == cost->ptr) return fail(ctx, TDV_ERR_INVALID_ARG, "aggreg aliases cost");
    }
    TDV_DEVICE_SCOPE(ctx);
    ctx->timer.begin(S(stream));
    return run_sgm(ctx, cost, guide, params, aggreg, out, S(stream));
}

tdv_status tdv_wta(tdv_ctx* ctx, const tdv_volume* vol, tdv_disparity* out, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_volume(ctx, vol, "vol", true));
    TDV_TRY(check_out(ctx, out));
    if (out->lr_threshold >= 0 || out->disp_right) {
        if (!out->disp) return fail(ctx, TDV_ERR_INVALID_ARG, "left-right check needs out->disp");
    }
    TDV_DEVICE_SCOPE(ctx);
    VolArg V = tdv::make_vol(*vol);
    ctx->timer.begin(S(stream));
    TDV_CUDA(tdv::launch_wta(V, out->disp, out->disp_norm, S(stream), &ctx->timer));
    if (out->lr_threshold >= 0 || out->disp_right)
        TDV_CUDA(tdv::launch_lr(V, out->disp, out->disp_norm, out->disp_right,
                                out->lr_threshold >= 0 ? out->lr_threshold : 0x7FFFFFFF, S(stream),
                                &ctx->timer));
    return TDV_OK;
}

tdv_status tdv_dp_scanline(tdv_ctx* ctx, const tdv_volume* cost, tdv_disparity* out,
                           tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_volume(ctx, cost, "cost", true));
    TDV_TRY(check_out(ctx, out));
    if (cost->depth > tdv::kMaxDispWide)
        return fail(ctx, TDV_ERR_UNSUPPORTED, "DP supports D <= %d (got %d)", tdv::kMaxDispWide,
                    cost->depth);
    if (out->lr_threshold >= 0 || out->disp_right)
        return fail(ctx, TDV_ERR_UNSUPPORTED, "DP has no left-right check");
    TDV_DEVICE_SCOPE(ctx);
    const size_t cb = (size_t)cost->width * cost->height * cost->depth;
    TDV_TRY(ensure(ctx, ctx->codes, cb));
    ctx->timer.begin(S(stream));
    TDV_CUDA(tdv::launch_dp(tdv::make_vol(*cost), out->disp, out->disp_norm, ctx->codes.ptr, cb,
                            S(stream), &ctx->timer));
    return TDV_OK;
}

tdv_status tdv_fast_wta(tdv_ctx* ctx, const tdv_image* left, const tdv_image* right, int32_t D,
                        int32_t radius, tdv_disparity* out, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_image(ctx, left, "left"));
    TDV_TRY(check_image(ctx, right, "right"));
    TDV_TRY(check_out(ctx, out));
    if (D <= 0 || D > 65535) return fail(ctx, TDV_ERR_INVALID_ARG, "bad max_disp %d", D);
    if (radius < 0 || radius > 15) return fail(ctx, TDV_ERR_INVALID_ARG, "bad radius %d", radius);
    if (out->lr_threshold >= 0 || out->disp_right)
        return fail(ctx, TDV_ERR_UNSUPPORTED, "fast WTA has no left-right check");
    if (left->width != right->width || left->height != right->height)
        return fail(ctx, TDV_ERR_INVALID_ARG, "left and right images differ in size");
    TDV_DEVICE_SCOPE(ctx);
    ctx->timer.begin(S(stream));
    TDV_CUDA(tdv::launch_fast_wta(tdv::make_img(*left), tdv::make_img(*right), D, radius, out->disp,
                                  out->disp_norm, S(stream), &ctx->timer));
    return TDV_OK;
}

tdv_status tdv_stereo_sgm(tdv_ctx* ctx, const tdv_image* left, const tdv_image* right, int32_t D,
                          const tdv_sgm_params* params, tdv_disparity* out, tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    TDV_TRY(check_image(ctx, left, "left"));
    TDV_TRY(check_image(ctx, right, "right"));
    TDV_TRY(check_params(ctx, params));
    TDV_TRY(check_out(ctx, out));
    if (D <= 0 || D > tdv::kMaxDispSgm)
        return fail(ctx, TDV_ERR_UNSUPPORTED, "SGM supports 1 <= D <= %d (got %d)", tdv::kMaxDispSgm, D);
    if (left->width != right->width || left->height != right->height)
        return fail(ctx, TDV_ERR_INVALID_ARG, "left and right images differ in size");
    const int W = left->width, H = left->height;
    ctx->timer.begin(S(stream));
    const FusedPlan fp = plan_fused(left, right, D, params);
    bool fused = fp.ok;
    TDV_DEVICE_SCOPE(ctx);
    if (fused && fp.weighted) {
        tdv_status werr;
        fused = fused_weights_ready(ctx, W, H, D, params, fp, S(stream), &werr);
        TDV_TRY(werr);
    }
    if (fused) {
        TDV_TRY(reserve_fused(ctx, W, H, D));
        TDV_TRY(ensure_side(ctx));
        TDV_TRY(ensure_err(ctx, S(stream)));
        tdv::FusedArgs a = fused_args(ctx, left, right, D, params, fp, out);
        a.planes = ctx->planes.ptr;
        a.agg = ctx->agg.ptr;
        a.agg2 = ctx->agg2.ptr;
        if (fp.weighted) a.side = (uint32_t*)ctx->fside.ptr;
        a.side_stream = ctx->side;
        a.fork = ctx->fork_ev;
        a.join = ctx->join_ev;
        TDV_CUDA(tdv::launch_fused(a, S(stream), &ctx->timer));
        return TDV_OK;
    }
    // general path: BT cost DSI into scratch, then the float aggregation
    TDV_TRY(ensure(ctx, ctx->cost, (size_t)W * H * D * sizeof(float)));
    tdv_volume cv;
    cv.ptr = ctx->cost.ptr;
    cv.width = W;
    cv.height = H;
    cv.depth = D;
    cv.layout = TDV_LAYOUT_HWD;
    cv.dtype = TDV_F32;
    TDV_CUDA(tdv::launch_cost(tdv::make_img(*left), tdv::make_img(*right), TDV_COST_BT, 0,
                              tdv::make_vol(cv), S(stream), &ctx->timer));
    return run_sgm(ctx, &cv, left, params, nullptr, out, S(stream));
}

tdv_status tdv_stereo_sgm_frames(tdv_ctx* ctx, int32_t n, const tdv_image* left, const tdv_image* right,
                                 int32_t D, const tdv_sgm_params* params, tdv_disparity* out,
                                 tdv_stream stream) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    if (n < 1 || !left || !right || !out) return fail(ctx, TDV_ERR_INVALID_ARG, "need n >= 1 frames and arrays");
    TDV_TRY(check_params(ctx, params));
    if (D <= 0 || D > tdv::kMaxDispSgm)
        return fail(ctx, TDV_ERR_UNSUPPORTED, "SGM supports 1 <= D <= %d (got %d)", tdv::kMaxDispSgm, D);
    const int W = left[0].width, H = left[0].height;
    FusedPlan fp;
    for (int i = 0; i < n; i++) {
        TDV_TRY(check_image(ctx, &left[i], "left"));
        TDV_TRY(check_image(ctx, &right[i], "right"));
        TDV_TRY(check_out(ctx, &out[i]));
        if (left[i].width != W || left[i].height != H || right[i].width != W || right[i].height != H)
            return fail(ctx, TDV_ERR_INVALID_ARG, "frame %d differs in size from frame 0", i);
        const FusedPlan f = plan_fused(&left[i], &right[i], D, params);
        if (!f.ok)
            return fail(ctx, TDV_ERR_UNSUPPORTED,
                        "frame sequences take the fused path only (u8 images at scale 1, P1/P2 multiples of "
                        "1/2, P2_CONST)");
        if (i == 0) fp = f;
    }
    TDV_DEVICE_SCOPE(ctx);
    cudaStream_t st = S(stream);
    if (fp.weighted) {
        tdv_status werr;
        const bool ok = fused_weights_ready(ctx, W, H, D, params, fp, st, &werr);
        TDV_TRY(werr);
        if (!ok)
            return fail(ctx, TDV_ERR_UNSUPPORTED, "this size, table and semantics leave the fused path's ranges");
    }
    TDV_TRY(reserve_fused(ctx, W, H, D));
    TDV_TRY(ensure_side(ctx));
    TDV_TRY(ensure_err(ctx, st));
    if (n > 1) {
        TDV_TRY(ensure_lane(ctx));
        TDV_TRY(ensure(ctx, ctx->planes_b, tdv::fused_plane_bytes(W, H)));
        TDV_TRY(ensure(ctx, ctx->agg_b, tdv::fused_agg_bytes(W, H, D)));
        TDV_TRY(ensure(ctx, ctx->agg2_b, tdv::fused_agg_bytes(W, H, D)));
        if (fp.weighted && ctx->fside.bytes) TDV_TRY(ensure(ctx, ctx->fside_b, ctx->fside.bytes));
        // the second lane starts after what the call's stream holds
        TDV_CUDA(cudaEventRecord(ctx->lane_start, st));
        TDV_CUDA(cudaStreamWaitEvent(ctx->lane_main, ctx->lane_start, 0));
    }
    for (int i = 0; i < n; i++) {
        tdv::FusedArgs a = fused_args(ctx, &left[i], &right[i], D, params, fp, &out[i]);
        const bool b = (i & 1) != 0;
        a.planes = b ? ctx->planes_b.ptr : ctx->planes.ptr;
        a.agg = b ? ctx->agg_b.ptr : ctx->agg.ptr;
        a.agg2 = b ? ctx->agg2_b.ptr : ctx->agg2.ptr;
        if (fp.weighted) a.side = (uint32_t*)(b ? ctx->fside_b.ptr : ctx->fside.ptr);
        a.side_stream = b ? ctx->lane_side : ctx->side;
        a.fork = b ? ctx->lane_fork : ctx->fork_ev;
        a.join = b ? ctx->lane_join : ctx->join_ev;
        TDV_CUDA(tdv::launch_fused(a, b ? ctx->lane_main : st, nullptr));
    }
    if (n > 1) {
        // the call's stream continues once the second lane is done
        TDV_CUDA(cudaEventRecord(ctx->lane_done, ctx->lane_main));
        TDV_CUDA(cudaStreamWaitEvent(st, ctx->lane_done, 0));
    }
    return TDV_OK;
}

// ------------------------------------------------------------ batched pairs
}  // extern "C"

struct tdv_batch {
    tdv_ctx* ctx = nullptr;
    std::vector<tdv::BatchPairArgs> pairs;
    int p1h = 0, p2h = 0, paths = 8;
    tdv_batch_tiles tiles{};
    tdv::BatchPlan plan;
    void* scratch = nullptr;
    void* desc = nullptr;
    size_t desc_bytes = 0;
    cudaGraphExec_t gexec = nullptr;
    unsigned long long wait_ns = 2000000000ull;
    int grid = 0;
    unsigned long long* trace = nullptr;  // caller's device buffer, 4 words per item, or null
};

namespace {

void* dev_alloc(tdv_ctx* ctx, size_t bytes) {
    void* p = nullptr;
    if (ctx->alloc) return ctx->alloc(bytes, ctx->alloc_user);
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void dev_free(tdv_ctx* ctx, void* p) {
    if (!p) return;
    if (ctx->release) ctx->release(p, ctx->alloc_user);
    else cudaFree(p);
}

void drop_graph(tdv_batch* b) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
}

// Plans with `t` and uploads the queue; the device must be idle for this
// batch (callers synchronise first).
tdv_status batch_replan(tdv_batch* b, const tdv_batch_tiles& t) {
    tdv_ctx* ctx = b->ctx;
    for (int pass = 0; pass < 2; pass++) {
        tdv::BatchPlan plan;
        const char* msg = tdv::batch_plan(b->pairs, b->p1h, b->p2h, b->paths, t, (unsigned char*)b->scratch,
                                          (unsigned char*)b->desc, plan);
        if (msg) return fail(ctx, TDV_ERR_UNSUPPORTED, "batch tiles: %s", msg);
        if (plan.bytes > b->desc_bytes) {
            // the descriptors hold the queue's own address: grow, then plan again
            dev_free(ctx, b->desc);
            b->desc = dev_alloc(ctx, plan.bytes);
            b->desc_bytes = b->desc ? plan.bytes : 0;
            if (!b->desc) return fail(ctx, TDV_ERR_OOM, "allocating %zu bytes of work queue failed", plan.bytes);
            continue;
        }
        TDV_CUDA(cudaMemcpy(b->desc, plan.desc.data(), plan.bytes, cudaMemcpyHostToDevice));
        b->plan = std::move(plan);
        b->tiles = t;
        drop_graph(b);
        return TDV_OK;
    }
    return fail(ctx, TDV_ERR_OOM, "work queue did not settle");
}

tdv_status batch_launch_on(tdv_batch* b, cudaStream_t st) {
    tdv_ctx* ctx = b->ctx;
    TDV_CUDA(tdv::batch_configure(b->plan));
    TDV_CUDA(tdv::batch_launch(b->plan, (unsigned char*)b->desc, b->wait_ns, b->grid, st, b->trace));
    return TDV_OK;
}

}  // namespace

extern "C" {

tdv_status tdv_batch_create(tdv_ctx* ctx, const tdv_batch_pair* pairs, int32_t n_pairs,
                            const tdv_sgm_params* params, tdv_batch** out) {
    if (!ctx) return TDV_ERR_INVALID_ARG;
    if (!out) return fail(ctx, TDV_ERR_INVALID_ARG, "null output handle");
    *out = nullptr;
    if (!pairs || n_pairs < 1 || n_pairs > 65536)
        return fail(ctx, TDV_ERR_INVALID_ARG, "n_pairs must be in [1, 65536] with a pair array");
    TDV_TRY(check_params(ctx, params));
    if (params->semantics != TDV_SEM_STANDARD || params->table != TDV_TABLE_FULL ||
        params->p2_mode != TDV_P2_CONST || !is_half_multiple(params->p1) || !is_half_multiple(params->p2) ||
        2.0f * params->p2 > 2560.0f)
        return fail(ctx, TDV_ERR_UNSUPPORTED,
                    "batches run the integer-domain fused path: STANDARD, FULL, P2_CONST, "
                    "P1/P2 multiples of 1/2, P2 <= 1280");
    std::vector<tdv::BatchPairArgs> args((size_t)n_pairs);
    for (int i = 0; i < n_pairs; i++) {
        const tdv_batch_pair& p = pairs[i];
        char nm[32];
        snprintf(nm, sizeof(nm), "pair %d left", i);
        TDV_TRY(check_image(ctx, &p.left, nm));
        snprintf(nm, sizeof(nm), "pair %d right", i);
        TDV_TRY(check_image(ctx, &p.right, nm));
        TDV_TRY(check_out(ctx, &p.out));
        if (p.left.dtype != TDV_U8 || p.right.dtype != TDV_U8 || p.left.scale != 1.0f || p.right.scale != 1.0f)
            return fail(ctx, TDV_ERR_UNSUPPORTED, "pair %d: batches take u8 images with scale 1", i);
        if (p.left.width != p.right.width || p.left.height != p.right.height)
            return fail(ctx, TDV_ERR_INVALID_ARG, "pair %d: left and right images differ in size", i);
        if (p.max_disp < 1 || p.max_disp > tdv::kMaxDispSgm)
            return fail(ctx, TDV_ERR_UNSUPPORTED, "pair %d: max_disp must be in [1, %d]", i, tdv::kMaxDispSgm);
        tdv::BatchPairArgs& a = args[i];
        a.L = tdv::make_img(p.left);
        a.R = tdv::make_img(p.right);
        a.W = p.left.width;
        a.H = p.left.height;
        a.D = p.max_disp;
        a.disp = p.out.disp;
        a.disp_norm = p.out.disp_norm;
        a.disp_right = p.out.disp_right;
        a.lr_thr = p.out.lr_threshold >= 0 ? p.out.lr_threshold : (p.out.disp_right ? 0x7FFFFFFF : -1);
    }
    TDV_DEVICE_SCOPE(ctx);
    tdv_batch* b = new (std::nothrow) tdv_batch;
    if (!b) return fail(ctx, TDV_ERR_OOM, "host allocation failed");
    b->ctx = ctx;
    b->pairs = std::move(args);
    b->p1h = (int)(2.0f * params->p1);
    b->p2h = (int)(2.0f * params->p2);
    b->paths = params->paths;
    if (cudaDeviceGetAttribute(&b->grid, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess ||
        b->grid < 1) {
        delete b;
        return fail(ctx, TDV_ERR_CUDA, "querying the SM count failed");
    }
    const size_t sb = tdv::batch_scratch_bytes(b->pairs);
    b->scratch = dev_alloc(ctx, sb);
    if (!b->scratch) {
        delete b;
        return fail(ctx, TDV_ERR_OOM, "allocating %zu bytes of batch scratch failed", sb);
    }
    tdv_batch_tiles t;
    t.lines_per_cta = 24;
    t.rows_per_cta = 8;
    t.split_disparity = 0;
    t.order = TDV_BATCH_ORDER_LONGEST_FIRST;
    t.ctas_per_sm = 1;
    const tdv_status st = batch_replan(b, t);
    if (st != TDV_OK) {
        tdv_batch_destroy(b);
        return st;
    }
    *out = b;
    return TDV_OK;
}

void tdv_batch_destroy(tdv_batch* b) {
    if (!b) return;
    DeviceScope ds(b->ctx->device);
    cudaDeviceSynchronize();
    drop_graph(b);
    dev_free(b->ctx, b->scratch);
    dev_free(b->ctx, b->desc);
    delete b;
}

tdv_status tdv_batch_set_tiles(tdv_batch* b, const tdv_batch_tiles* tiles) {
    if (!b) return TDV_ERR_INVALID_ARG;
    tdv_ctx* ctx = b->ctx;
    if (!tiles) return fail(ctx, TDV_ERR_INVALID_ARG, "null tiles");
    if (tiles->order != TDV_BATCH_ORDER_LONGEST_FIRST && tiles->order != TDV_BATCH_ORDER_INPUT)
        return fail(ctx, TDV_ERR_INVALID_ARG, "bad queue order %d", tiles->order);
    if (tiles->split_disparity != 0 && tiles->split_disparity != 1)
        return fail(ctx, TDV_ERR_INVALID_ARG, "split_disparity must be 0 or 1");
    if (tiles->ctas_per_sm != 1 && tiles->ctas_per_sm != 2)
        return fail(ctx, TDV_ERR_INVALID_ARG, "ctas_per_sm must be 1 or 2");
    TDV_DEVICE_SCOPE(ctx);
    TDV_CUDA(cudaDeviceSynchronize());
    return batch_replan(b, *tiles);
}

tdv_status tdv_batch_get_tiles(const tdv_batch* b, tdv_batch_tiles* tiles) {
    if (!b || !tiles) return TDV_ERR_INVALID_ARG;
    *tiles = b->tiles;
    return TDV_OK;
}

tdv_status tdv_batch_run(tdv_batch* b, tdv_stream stream) {
    if (!b) return TDV_ERR_INVALID_ARG;
    tdv_ctx* ctx = b->ctx;
    TDV_DEVICE_SCOPE(ctx);
    return batch_launch_on(b, S(stream));
}

tdv_status tdv_batch_graph_launch(tdv_batch* b, tdv_stream stream) {
    if (!b) return TDV_ERR_INVALID_ARG;
    tdv_ctx* ctx = b->ctx;
    TDV_DEVICE_SCOPE(ctx);
    if (!b->gexec) {
        // the shared-memory opt-in is not a stream operation: set it outside the capture
        TDV_CUDA(tdv::batch_configure(b->plan));
        cudaStream_t cs;
        TDV_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            const cudaError_t el =
                tdv::batch_launch(b->plan, (unsigned char*)b->desc, b->wait_ns, b->grid, cs, b->trace);
            e = cudaStreamEndCapture(cs, &g);
            if (el != cudaSuccess) e = el;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->gexec, g, 0);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) {
            b->gexec = nullptr;
            return fail(ctx, TDV_ERR_CUDA, "capturing the batch graph failed: %s", cudaGetErrorString(e));
        }
    }
    TDV_CUDA(cudaGraphLaunch(b->gexec, S(stream)));
    return TDV_OK;
}

tdv_status tdv_batch_status(tdv_batch* b, tdv_stream stream) {
    if (!b) return TDV_ERR_INVALID_ARG;
    tdv_ctx* ctx = b->ctx;
    TDV_DEVICE_SCOPE(ctx);
    TDV_CUDA(cudaStreamSynchronize(S(stream)));
    int w[2] = {0, 0};
    TDV_CUDA(cudaMemcpy(w, (unsigned char*)b->desc + b->plan.ctl_off, sizeof(w), cudaMemcpyDeviceToHost));
    if (w[1] == TDV_ERR_TIMEOUT)
        return fail(ctx, TDV_ERR_TIMEOUT, "a bounded wait in the batch kernel ran out");
    if (w[1] == TDV_ERR_BAD_WORK)
        return fail(ctx, TDV_ERR_BAD_WORK, "the batch work queue held an item out of range");
    if (w[1] != 0) return fail(ctx, TDV_ERR_CUDA, "batch kernel recorded status %d", w[1]);
    return TDV_OK;
}

tdv_status tdv_batch_set_wait_limit(tdv_batch* b, double seconds) {
    if (!b) return TDV_ERR_INVALID_ARG;
    if (!(seconds >= 1e-3 && seconds <= 60.0))
        return fail(b->ctx, TDV_ERR_INVALID_ARG, "wait limit must be in [0.001, 60] s");
    b->wait_ns = (unsigned long long)(seconds * 1e9);
    drop_graph(b);
    return TDV_OK;
}

tdv_status tdv_batch_set_trace(tdv_batch* b, unsigned long long* trace, int64_t capacity_items) {
    if (!b) return TDV_ERR_INVALID_ARG;
    if (trace && capacity_items < b->plan.n_items)
        return fail(b->ctx, TDV_ERR_INVALID_ARG, "trace holds %lld items, the queue %d", (long long)capacity_items,
                    b->plan.n_items);
    b->trace = trace;
    drop_graph(b);
    return TDV_OK;
}

tdv_status tdv_batch_work_queue(tdv_batch* b, void** items, int32_t* n_items, int32_t* item_bytes) {
    if (!b) return TDV_ERR_INVALID_ARG;
    if (!items || !n_items || !item_bytes) return fail(b->ctx, TDV_ERR_INVALID_ARG, "null output");
    *items = (unsigned char*)b->desc + b->plan.items_off;
    *n_items = b->plan.n_items;
    *item_bytes = b->plan.item_bytes;
    return TDV_OK;
}

tdv_status tdv_batch_autotune(tdv_batch* b, int32_t reps, tdv_stream stream, tdv_batch_tiles* chosen,
                              double* best_ms) {
    if (!b) return TDV_ERR_INVALID_ARG;
    tdv_ctx* ctx = b->ctx;
    if (reps < 1 || reps > 100) return fail(ctx, TDV_ERR_INVALID_ARG, "reps must be in [1, 100]");
    TDV_DEVICE_SCOPE(ctx);
    cudaStream_t st = S(stream);
    cudaEvent_t e0, e1;
    TDV_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(ctx, TDV_ERR_CUDA, "cudaEventCreate failed");
    }
    // times one candidate; +inf if it does not fit
    auto time_tiles = [&](const tdv_batch_tiles& t, double& ms) -> tdv_status {
        ms = HUGE_VAL;
        TDV_CUDA(cudaStreamSynchronize(st));
        if (batch_replan(b, t) != TDV_OK) return TDV_OK;
        TDV_TRY(batch_launch_on(b, st));  // warm-up
        TDV_TRY(tdv_batch_status(b, stream));
        TDV_CUDA(cudaEventRecord(e0, st));
        for (int r = 0; r < reps; r++) TDV_TRY(batch_launch_on(b, st));
        TDV_CUDA(cudaEventRecord(e1, st));
        TDV_TRY(tdv_batch_status(b, stream));
        float f = 0.0f;
        TDV_CUDA(cudaEventElapsedTime(&f, e0, e1));
        ms = (double)f / reps;
        return TDV_OK;
    };
    tdv_batch_tiles best = b->tiles;
    double best_t = HUGE_VAL;
    tdv_status st_all = time_tiles(best, best_t);
    int wmax = 1, hmax = 1;
    for (const auto& p : b->pairs) {
        wmax = std::max(wmax, p.W);
        hmax = std::max(hmax, p.H);
    }
    // one coordinate descent per blocks-per-SM setting (it bounds the lines
    // and rows a block can take), over lines, rows, split and queue order;
    // besides fixed sizes, the sizes that give the largest pair one tile per
    // block slot
    for (int ctas = 1; ctas <= 2 && st_all == TDV_OK; ctas++) {
        tdv_batch_tiles cur = b->tiles;
        cur.ctas_per_sm = ctas;
        double cur_t;
        st_all = time_tiles(cur, cur_t);
        const int slots = ctas * b->grid;
        const int g_fit = std::min(24, std::max(1, (wmax + slots - 1) / slots));
        const int r_fit = std::min(24, std::max(1, (hmax + slots - 1) / slots));
        const int Gs[] = {8, 12, 16, 20, 24, g_fit};
        const int Rs[] = {4, 6, 8, 12, 16, 24, r_fit};
        for (int axis = 0; axis < 4 && st_all == TDV_OK; axis++) {
            const int n = axis == 0 ? 6 : (axis == 1 ? 7 : 2);
            for (int j = 0; j < n && st_all == TDV_OK; j++) {
                tdv_batch_tiles t = cur;
                if (axis == 0) t.lines_per_cta = Gs[j];
                else if (axis == 1) t.rows_per_cta = Rs[j];
                else if (axis == 2) t.split_disparity = j;
                else t.order = j;
                if (memcmp(&t, &cur, sizeof(t)) == 0) continue;
                double ms;
                st_all = time_tiles(t, ms);
                if (st_all == TDV_OK && ms < cur_t) {
                    cur_t = ms;
                    cur = t;
                }
            }
        }
        if (st_all == TDV_OK && cur_t < best_t) {
            best_t = cur_t;
            best = cur;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st_all != TDV_OK) return st_all;
    TDV_CUDA(cudaStreamSynchronize(st));
    TDV_TRY(batch_replan(b, best));
    if (chosen) *chosen = best;
    if (best_ms) *best_ms = best_t;
    return TDV_OK;
}

}  // extern "C"
