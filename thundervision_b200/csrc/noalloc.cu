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
//    address.  Set-up happens once per device and context: the first call on
//    a device (and the first after a device reset or in another context on
//    it, which may place the array elsewhere) looks the address up with
//    cudaGetSymbolAddress while that device is current and remembers it with
//    the context's id.  Make that first call before any stream capture: a
//    call whose stream is capturing cannot do the set-up and returns
//    TDV_ERR_INVALID_ARG instead.
//  * All calls share the one array and it keeps the previous call's contents.
//    Each call clears the error word; the planes and the aggregation volume
//    are completely written before they are read.  Calls whose GPU work
//    overlaps (other streams, other host threads) race on the array.
//  * Scratch: BT planes of 16*(W + 9*ceil(W/8)) bytes per row (about 34 B per
//    pixel), plus the volume of 128*ppl bytes per pixel (ppl = 1 for D <= 64,
//    2 for D <= 128, 4 for D <= 256), each rounded up to 256 bytes, plus
//    256 bytes for the error word.  Pairs that do not fit, and inputs outside
//    the fused path (not u8 with scale 1, non-STANDARD semantics, REF table,
//    adjusted P2, penalties that are not non-negative multiples of 1/2,
//    P2 > 1280, D > 256), are rejected with TDV_ERR_UNSUPPORTED before any GPU
//    work; malformed arguments (null pointers, non-finite penalties, values
//    outside the enums, left/right sizes that differ) with
//    TDV_ERR_INVALID_ARG.
//  * Every wait inside the kernels is bounded.  If one runs out (a copy that
//    never lands: a failing device), the call's last kernel marks every pixel
//    of every requested output invalid (0xFFFF, -1.0f), so a map is never
//    returned half-written; the call itself returns once its work is queued.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "tdv_internal.hpp"

namespace {

constexpr size_t kStaticScratchBytes = (size_t)64 << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Per device: the array's address and the id of the context it was resolved
// in (context ids are unique for the life of the process).
struct Resolved {
    unsigned long long ctx_id = 0;
    void* addr = nullptr;
};
std::mutex g_setup_mu;
Resolved g_scratch[kMaxDevices];

// The current context's id through the driver entry points (the library links
// only the runtime).  0 if the driver cannot tell.
unsigned long long current_context_id() {
    using GetCurrentFn = int (*)(void**);
    using GetIdFn = int (*)(void*, unsigned long long*);
    static GetCurrentFn get_current = nullptr;
    static GetIdFn get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess && f)
            get_current = (GetCurrentFn)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess && f)
            get_id = (GetIdFn)f;
        cudaGetLastError();
        looked_up = true;
    }
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

size_t round256(size_t v) { return (v + 255) & ~(size_t)255; }

bool half_multiple(float v) { return v >= 0.0f && v <= 4096.0f && std::floor(2.0f * v) == 2.0f * v; }

bool image_ok(const tdv_image* im) {
    return im->width > 0 && im->height > 0 && im->width <= 16384 && im->height <= 16384 &&
           im->pitch >= im->width && im->dtype == TDV_U8 && im->scale == 1.0f;
}

// After the fused kernels: if one of them recorded a failed wait, every pixel
// of the requested outputs is marked invalid.
__global__ void mark_failed_kernel(const int* err, int n, uint16_t* disp, float* disp_norm, uint16_t* disp_right) {
    if (*(volatile const int*)err == 0) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (disp) disp[i] = 0xFFFF;
        if (disp_norm) disp_norm[i] = -1.0f;
        if (disp_right) disp_right[i] = 0xFFFF;
    }
}

}  // namespace

extern "C" tdv_status tdv_stereo_sgm_static(const tdv_image* left, const tdv_image* right, int32_t max_disp,
                                            const tdv_sgm_params* params, tdv_disparity* out,
                                            tdv_stream stream) {
    if (!left || !right || !params || !out || !left->ptr || !right->ptr) return TDV_ERR_INVALID_ARG;
    if (!out->disp && !out->disp_norm && !out->disp_right) return TDV_ERR_INVALID_ARG;
    if (!std::isfinite(params->p1) || !std::isfinite(params->p2)) return TDV_ERR_INVALID_ARG;
    if (params->p2_mode != TDV_P2_CONST && params->p2_mode != TDV_P2_ADJUST) return TDV_ERR_INVALID_ARG;
    if (params->table != TDV_TABLE_FULL && params->table != TDV_TABLE_REF) return TDV_ERR_INVALID_ARG;
    if (params->semantics < TDV_SEM_STANDARD || params->semantics > TDV_SEM_REF_GPU) return TDV_ERR_INVALID_ARG;
    if (params->paths != 4 && params->paths != 8) return TDV_ERR_INVALID_ARG;
    if (left->width != right->width || left->height != right->height) return TDV_ERR_INVALID_ARG;
    if (!image_ok(left) || !image_ok(right)) return TDV_ERR_UNSUPPORTED;
    if (max_disp <= 0 || max_disp > tdv::kMaxDispSgm) return TDV_ERR_UNSUPPORTED;
    if (params->semantics != TDV_SEM_STANDARD || params->table != TDV_TABLE_FULL ||
        params->p2_mode != TDV_P2_CONST || !half_multiple(params->p1) || !half_multiple(params->p2) ||
        2.0f * params->p2 > 2560.0f)
        return TDV_ERR_UNSUPPORTED;

    const int W = left->width, H = left->height;
    const size_t plane_bytes = round256(tdv::fused_plane_bytes(W, H));
    const size_t agg_bytes = round256(tdv::fused_agg_bytes(W, H, max_disp));
    if (plane_bytes + agg_bytes + 256 > kStaticScratchBytes) return TDV_ERR_UNSUPPORTED;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return TDV_ERR_CUDA;
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
        cudaGetLastError();
        return TDV_ERR_CUDA;
    }
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        Resolved& r = g_scratch[dev];
        const unsigned long long id = current_context_id();
        if (!r.addr || id == 0 || id != r.ctx_id) {
            // set-up: not possible while the stream is being captured
            if (cap != cudaStreamCaptureStatusNone) return TDV_ERR_INVALID_ARG;
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return TDV_ERR_CUDA;
            }
            r.addr = p;
            r.ctx_id = id;
        }
        base = r.addr;
    }
    unsigned char* b = (unsigned char*)base;
    int* err = (int*)(b + plane_bytes + agg_bytes);
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
    if (tdv::launch_fused(a, st, nullptr) != cudaSuccess) return TDV_ERR_CUDA;
    const int n = W * H;
    mark_failed_kernel<<<(n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184, 256, 0, st>>>(err, n, out->disp,
                                                                                        out->disp_norm,
                                                                                        out->disp_right);
    return cudaGetLastError() == cudaSuccess ? TDV_OK : TDV_ERR_CUDA;
}
