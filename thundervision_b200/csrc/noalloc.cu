// tdv_stereo_sgm_static: the fused BT + SGM + WTA path for callers that must
// not allocate device memory.
//
// Some callers of this library cannot call cudaMalloc (or any routine that
// allocates) at the point where they run stereo matching: a camera or robot
// control loop whose device memory is budgeted once at start-up, a plugin
// hosted by an application that owns every device allocation, or a real-time
// frame loop where an allocation could stall past its deadline.  For them this
// entry point runs the same kernels as tdv_stereo_sgm's fused integer-domain
// path, with every piece of scratch (the BT planes, the 16-bit aggregation
// volume and the device error word) carved from one file-scope __device__
// array of kStaticScratchBytes.  The caller still passes the input images and
// the output buffers; no context is involved.
//
// What a caller must know:
//  * The array belongs to this library's device code: every GPU on which the
//    library's module is loaded holds kStaticScratchBytes (64 MiB) of device
//    memory until the process exits.
//  * In host code the array's name is only a host-side stand-in, not a device
//    address.  The first call on each device looks the address up with
//    cudaGetSymbolAddress while that device is current and caches it, so make
//    the first call on a device before any stream capture starts.
//  * All calls share the one array and it keeps the previous call's contents.
//    Each call clears the error word; the planes and the aggregation volume
//    are completely written before they are read.  Calls whose GPU work
//    overlaps (other streams, other host threads) race on the array.
//  * Pairs whose scratch does not fit (BT planes ~34 B/pixel + the volume
//    128*ceil(D/64) B/pixel + 256 B), and inputs outside the fused path (not
//    u8 with scale 1, non-STANDARD semantics, REF table, adjusted P2,
//    penalties that are not non-negative multiples of 1/2, P2 > 1280,
//    D > 256, left/right sizes that differ), are rejected with
//    TDV_ERR_UNSUPPORTED or TDV_ERR_INVALID_ARG before any GPU work.
//  * A bounded wait that runs out inside the kernels is recorded in the error
//    word but not reported by this call, which returns once its work is
//    queued.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "tdv_internal.hpp"

namespace {

constexpr size_t kStaticScratchBytes = (size_t)64 << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

size_t round256(size_t v) { return (v + 255) & ~(size_t)255; }

bool half_multiple(float v) { return v >= 0.0f && v <= 4096.0f && std::floor(2.0f * v) == 2.0f * v; }

bool image_ok(const tdv_image* im) {
    return im && im->ptr && im->width > 0 && im->height > 0 && im->width <= 16384 &&
           im->height <= 16384 && im->pitch >= im->width && im->dtype == TDV_U8 && im->scale == 1.0f;
}

}  // namespace

extern "C" tdv_status tdv_stereo_sgm_static(const tdv_image* left, const tdv_image* right, int32_t max_disp,
                                            const tdv_sgm_params* params, tdv_disparity* out,
                                            tdv_stream stream) {
    if (!left || !right || !params || !out) return TDV_ERR_INVALID_ARG;
    if (!out->disp && !out->disp_norm && !out->disp_right) return TDV_ERR_INVALID_ARG;
    if (!image_ok(left) || !image_ok(right)) return TDV_ERR_UNSUPPORTED;
    if (left->width != right->width || left->height != right->height) return TDV_ERR_INVALID_ARG;
    if (max_disp <= 0 || max_disp > tdv::kMaxDispSgm) return TDV_ERR_UNSUPPORTED;
    if (params->paths != 4 && params->paths != 8) return TDV_ERR_INVALID_ARG;
    if (params->semantics != TDV_SEM_STANDARD || params->table != TDV_TABLE_FULL ||
        params->p2_mode != TDV_P2_CONST || !half_multiple(params->p1) || !half_multiple(params->p2) ||
        2.0f * params->p2 > 2560.0f)
        return TDV_ERR_UNSUPPORTED;

    const int W = left->width, H = left->height;
    const size_t plane_bytes = round256(tdv::fused_plane_bytes(W, H));
    const size_t agg_bytes = round256(tdv::fused_agg_bytes(W, H, max_disp));
    if (plane_bytes + agg_bytes + 256 > kStaticScratchBytes) return TDV_ERR_UNSUPPORTED;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TDV_ERR_CUDA;
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return TDV_ERR_CUDA;
            }
            g_scratch_addr[dev] = p;
        }
        base = g_scratch_addr[dev];
    }
    unsigned char* b = (unsigned char*)base;
    int* err = (int*)(b + plane_bytes + agg_bytes);
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return TDV_ERR_CUDA;

    tdv::FusedArgs a;
    a.L = tdv::make_img(*left);
    a.R = tdv::make_img(*right);
    a.W = W;
    a.H = H;
    a.D = max_disp;
    a.p1h = (int)(2.0f * params->p1);
    a.p2h = (int)(2.0f * params->p2);
    a.paths = params->paths;
    a.disp = out->disp;
    a.disp_norm = out->disp_norm;
    a.disp_right = out->disp_right;
    a.lr_thr = out->lr_threshold >= 0 ? out->lr_threshold : (out->disp_right ? 0x7FFFFFFF : -1);
    a.planes = b;
    a.agg = b + plane_bytes;
    a.err = err;
    return tdv::launch_fused(a, st, nullptr) == cudaSuccess ? TDV_OK : TDV_ERR_CUDA;
}
