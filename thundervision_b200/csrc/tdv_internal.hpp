// Internal declarations shared by the C-ABI host code and the kernel files.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/tdv_stereo.h"

namespace tdv {

// Largest disparity range handled by the SGM / WTA kernels (8 values per lane
// of one warp for fp32 paths = 256, the reference's SG_MAX_DISP,
// tdvision/semiglobal.cu:44; the DP and WTA kernels take up to 1024).
constexpr int kMaxDispSgm = 256;
constexpr int kMaxDispWide = 1024;

// One walk of an aggregation pass: start cell, number of cells, and how many
// identical walks the reference table issues back to back (REF tables repeat
// some reverse diagonals).  A repeated walk (mult > 1) stores its per-cell
// path costs in the deferred buffer, from row `defer` on (one row of D floats
// per step), and a second kernel adds each of them mult times into S.
struct Walk {
    int32_t sx, sy, len, mult, defer;
};

// An ordered aggregation pass: all walks share one direction and touch
// disjoint cells, so they run concurrently while every cell still sees the
// reference's per-cell order of updates.
struct Pass {
    int dx, dy;
    size_t first, count;    // range in the device walk array
    size_t dfirst, dcount;  // its repeated walks: range in the deferred index array
    int dmaxlen;            // longest repeated walk of the pass
};

struct PassSchedule {
    int W = 0, H = 0, table = -1, paths = 0;
    std::vector<Pass> passes;
    std::vector<Walk> walks;         // host copy
    std::vector<int32_t> deferred;   // indices (into walks) of repeated walks, pass by pass
    long long defer_rows = 0;        // deferred-buffer rows one pass needs at most
    Walk* d_walks = nullptr;         // device copies (ctx scratch)
    int32_t* d_deferred = nullptr;
};

// Optional per-kernel timing.  Every kernel of one ABI call is bracketed by
// CUDA events on the stream it runs on: an entry spans from the previous
// event recorded on that stream (the call's start, a fork, or the previous
// kernel there) to the event recorded after the kernel.
struct Timer {
    bool on = false;
    std::vector<cudaEvent_t> ev;
    std::vector<std::string> names;
    std::vector<std::pair<int, int>> spans;  // (start event, end event) per entry
    int n = 0;
    cudaStream_t st = nullptr, side = nullptr;
    int last_main = -1, last_side = -1;
    void begin(cudaStream_t s) {
        if (!on) return;
        n = 0;
        names.clear();
        spans.clear();
        st = s;
        side = nullptr;
        last_main = rec(s);
    }
    void mark(const char* name) { mark_on(name, st); }
    void mark_on(const char* name, cudaStream_t s) {
        if (!on) return;
        int& last = (s == st || s != side) ? last_main : last_side;
        const int e = rec(s);
        if (e < 0) return;
        names.emplace_back(name);
        spans.emplace_back(last, e);
        last = e;
    }
    // a second stream joined the call (after it waited on a fork event)
    void fork(cudaStream_t s) {
        if (!on) return;
        side = s;
        last_side = rec(s);
    }
    // the call's stream waited on the second stream's join event
    void join() {
        if (!on) return;
        last_main = rec(st);
    }
    int rec(cudaStream_t s) {
        if (n >= (int)ev.size()) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return -1;
            ev.push_back(e);
        }
        cudaEventRecord(ev[n], s);
        return n++;
    }
};

// Builds the reference's path table (tdvision/semiglobal.cu:57-230) or its
// corrected FULL variant and schedules it into passes; see paths.cpp.
// Returns false (and schedules nothing usable) if a walk leaves the image.
bool build_schedule(int W, int H, int table, int paths, PassSchedule& out);

// Walk weights of the fused path (paths.cpp).  The fused kernels walk every
// path line of each of the 8 directions exactly once, from the image edge it
// enters.  The reference's sequential loop over its table differs in ways
// that only change how many times a direction's path cost L_k(p) counts in
// S(p) = sum_k n_k(p) L_k(p): a stale table walks some reverse diagonals
// never and one of them many times, and with start-assign semantics
// (tdvision/semiglobalcpu.cpp:79-83) a walk starting at a border cell wipes
// what earlier walks added there.  n_k(p) is found by replaying the table's
// walk order on the host and stored compactly as weight classes:
//   0 = the cell does not count L_k, 1 = it counts once, 2 = it counts
//   n >= 2 times (only on the one "corner" line of the reverse diagonal
//   directions whose table ends are stale).
// Every line of a direction (a column, a diagonal or a row) has one class for
// its interior cells; a line whose border cells count otherwise carries the
// flag 4, and only flagged lines look up their border cells' classes.
// Fused direction order: V+ V- D1+ D1- D2+ D2- H+ H- with (dx, dy) =
// (0,1) (0,-1) (1,1) (-1,-1) (-1,1) (1,-1) (1,0) (-1,0); D1- and D2- are the
// corner slots 0 and 1.
constexpr int kFusedDirs = 8;
struct FusedWeights {
    int W = 0, H = 0, table = -1, paths = 0, assign = -1;
    bool has_line = false;    // some line is not all-ones (or is flagged)
    bool has_border = false;  // some border cells carry their own classes
    bool has_corner = false;  // some cell counts a direction more than once
    int max_wm1 = 0;          // largest n - 1 over the corner cells
    int nl = 0, nb = 0;       // line slots per direction (W + H - 1), border cells (2W + 2H)
    // device image: [8][nl] line classes (the horizontal directions indexed
    // by row), [8][nb] border classes, then per row two corner entries
    // (int32 x or -1, int32 (n-1) << 1 | slot)
    size_t lw_off = 0, bw_off = 0, corner_off = 0, bytes = 0;
    std::vector<unsigned char> image;
};
// Border cell index: row 0 -> x, row H-1 -> W + x, column 0 -> 2W + y,
// column W-1 -> 2W + H + y.
__host__ __device__ inline int border_index(int W, int H, int x, int y) {
    return y == 0 ? x : (y == H - 1 ? W + x : (x == 0 ? 2 * W + y : 2 * W + H + y));
}
// Returns false (with a reason) when the table's weights do not fit this
// model; the caller then takes the general path.
bool build_fused_weights(int W, int H, int table, int paths, bool assign, FusedWeights& out, const char** why);

}  // namespace tdv

struct tdv_ctx {
    int device = 0;
    bool device_set = false;
    std::string last_error;
    tdv_alloc_fn alloc = nullptr;
    tdv_free_fn release = nullptr;
    void* alloc_user = nullptr;

    // scratch buffers, grown on demand
    struct Buf {
        void* ptr = nullptr;
        size_t bytes = 0;
    };
    Buf agg;      // aggregation volume
    Buf agg2;     // fused path: second aggregation volume (concurrent pass chains)
    Buf cost;     // cost DSI for tdv_stereo_sgm's general path
    Buf planes;   // fused path: left/right BT planes
    Buf codes;    // DP choice codes
    Buf misc;     // small per-call scratch
    Buf err;      // one device int: error status written by kernels
    Buf soft;     // soft-SGM: dS volume / inference-mode S and statistics
    Buf defer;    // general SGM: path costs of repeated walks, one pass at a time
    std::vector<long long> ckpt_off_host;

    tdv::PassSchedule sched;
    Buf sched_buf;
    // fused path with the reference recurrence / table: walk weights of the
    // last size seen (host description and device image) and the side rows
    tdv::FusedWeights fweights;
    Buf fw_buf;
    Buf fside;
    tdv::Timer timer;
    // fused path: side stream and fork/join events of the two pass chains
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    // fused path over a frame sequence (tdv_stereo_sgm_frames): the second
    // lane's planes, volumes and side rows, its two streams, its chains'
    // fork/join events and the events that tie it to the call's stream
    Buf planes_b, agg_b, agg2_b, fside_b;
    cudaStream_t lane_main = nullptr, lane_side = nullptr;
    cudaEvent_t lane_fork = nullptr, lane_join = nullptr, lane_start = nullptr, lane_done = nullptr;
};

namespace tdv {

// ---- kernel launchers (defined in the .cu kernel files) ----------------

struct ImgArg {
    const void* ptr;
    int W, H, pitch;
    int u8;  // 1: uint8, 0: float
    float scale;
};

// A 2-D pixel array with interleaved channels (tdv_raster); pitch in bytes,
// dtype 0 = F32, 1 = U16, 2 = U8.
struct RasterArg {
    void* ptr;
    int W, H;
    long long pitch;
    int dtype, ch;
};

struct VolArg {
    void* ptr;
    int W, H, D;
    long long sx, sy;  // element strides of the pixel (x, y)
    int u16 = 0;       // 1: TDV_U16 cost in half-units (0xFFFF = +INF), else float elements
};

VolArg make_vol(const tdv_volume& v);
ImgArg make_img(const tdv_image& im);

cudaError_t launch_cost(const ImgArg& L, const ImgArg& R, int kind, int radius, const VolArg& out,
                        cudaStream_t st, Timer* tm);
// banded cost kernels (kernels_cost.cu): BT, and SSD / NCC with radius 1..4;
// `prefiltered` fuses the 5x5 Gaussian of both images into the band staging
// and writes the filtered left image (DSI width x height) when left_filtered
// is not null
bool cost_banded_supported(int kind, int radius, int D, bool prefiltered = false);
cudaError_t launch_cost_banded(const ImgArg& L, const ImgArg& R, int kind, int radius, const VolArg& out,
                               bool prefiltered, float* left_filtered, cudaStream_t st);
// FastWTA on the banded SSD (radius 1..4, bands within the cost kernels' budget)
cudaError_t launch_fast_wta_banded(const ImgArg& L, const ImgArg& R, int D, int radius, uint16_t* disp,
                                  float* disp_norm, cudaStream_t st);

struct SgmArgs {
    VolArg C, S;
    ImgArg guide;
    int has_guide;
    float p1, p2;
    int p2_adjust, sem;
    float* defer;  // path costs of the repeated walks of one pass (PassSchedule::defer_rows x D)
};
cudaError_t launch_sgm_passes(const SgmArgs& a, const PassSchedule& sch, cudaStream_t st, Timer* tm);
cudaError_t launch_wta(const VolArg& V, uint16_t* disp, float* disp_norm, cudaStream_t st, Timer* tm);
cudaError_t launch_lr(const VolArg& S, uint16_t* dispL, float* disp_norm, uint16_t* dispR,
                      int thr, cudaStream_t st, Timer* tm);
cudaError_t launch_dp(const VolArg& C, uint16_t* disp, float* disp_norm, void* codes_scratch,
                      size_t codes_bytes, cudaStream_t st, Timer* tm);
cudaError_t launch_fast_wta(const ImgArg& L, const ImgArg& R, int D, int radius, uint16_t* disp,
                            float* disp_norm, cudaStream_t st, Timer* tm);

// Fused integer-domain BT + SGM + WTA (+ left-right check).
struct FusedArgs {
    ImgArg L, R;
    int W, H, D;
    int p1h, p2h;  // penalties in half-units (2*P)
    int paths;
    uint16_t* disp;
    float* disp_norm;
    uint16_t* disp_right;
    int lr_thr;
    void* planes;  // fused_plane_bytes(W, H)
    void* agg;     // fused_agg_bytes(W, H, D)
    int* err;      // device word: kernels record TDV_ERR_TIMEOUT here
    // Optional second aggregation volume and stream: with both (8 paths),
    // the passes run as two concurrent chains, V+ V- D1+ into `agg` on the
    // call's stream and D1- D2+ D2- into `agg2` on `side`; H+ joins them
    // (agg += agg2 + its L) and H- finishes agg.
    void* agg2 = nullptr;
    cudaStream_t side_stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    // The reference recurrences and table (see fused_body.cuh): `excl` leaves
    // d = D-1 out of the minimum, `gstart` starts a line the reference GPU
    // recurrence's way, `off_h` is the per-direction offset in
    // half-units, `weights` the device image of `fw` (null: every cell counts
    // every direction once), `side` 2 * H * fused_side_words(D) words of
    // repeated-line rows when fw->has_corner.
    int excl = 0;
    int off_h = 0;
    int gstart = 0;  // the reference GPU recurrence: P1 in half-units, else 0
    const unsigned char* weights = nullptr;
    const FusedWeights* fw = nullptr;
    uint32_t* side = nullptr;
};
size_t fused_agg_bytes(int W, int H, int D);
// 32-bit words of one repeated-line side row (a pixel's S vector).
inline size_t fused_side_words(int D) { return (size_t)32 * (D <= 64 ? 1 : (D <= 128 ? 2 : 4)); }

// Image stages either side of the path (kernels_image.cu).
cudaError_t launch_to_gray(const RasterArg& color, float* gray, cudaStream_t st);
// K row-major 3x3, dist (k1 k2 p1 p2 k3 k4 k5 k6), iR = inv(P[:, :3] R) row-major
cudaError_t launch_rectify_maps(const double* K, const double* dist, const double* iR, int W, int H, float* mapx,
                               float* mapy, cudaStream_t st);
cudaError_t launch_remap(const RasterArg& src, const float* mx, const float* my, const RasterArg& dst,
                         cudaStream_t st);
cudaError_t launch_prefilter(const ImgArg& in, int kind, float* out, cudaStream_t st);
// kind 0 (opening) needs `scratch` of W*H elements of the map's dtype
cudaError_t launch_postfilter(const RasterArg& in, int kind, const RasterArg& out, void* scratch,
                              cudaStream_t st);
cudaError_t launch_subpixel(const float* S, int W, int H, int D, const uint16_t* disp, float* out,
                            cudaStream_t st);
cudaError_t launch_reproject(const RasterArg& disp, const RasterArg* color, int mode, float zscale,
                             const float* q, float* verts, float* cols, cudaStream_t st);
size_t fused_plane_bytes(int W, int H);
cudaError_t launch_fused(const FusedArgs& a, cudaStream_t st, Timer* tm);

// Batched fused path (kernels_batch.cu): one persistent launch for many
// integer-domain pairs of uneven size and disparity range.
struct BatchPairArgs {
    ImgArg L, R;
    int W, H, D;
    uint16_t* disp;
    float* disp_norm;
    uint16_t* disp_right;
    int lr_thr;
};
using BatchTiles = tdv_batch_tiles;
// Device image of the plan: [control words][pair descriptors][work items].
struct BatchPlan {
    std::vector<unsigned char> desc;
    size_t ctl_off = 0, pairs_off = 0, items_off = 0, bytes = 0;
    int n_pairs = 0, n_items = 0, smem = 0, item_bytes = 0, ctas_per_sm = 1;
};
int batch_passes();
int batch_threads();
size_t batch_ctl_bytes(int npairs);
// planes + aggregation volumes of all pairs, each 256-byte aligned
size_t batch_scratch_bytes(const std::vector<BatchPairArgs>& pairs);
// Builds the plan for scratch at `scratch` and the descriptor copy at
// `d_desc` (device addresses, used only to fill pointers); returns an error
// message, or nullptr on success.
const char* batch_plan(const std::vector<BatchPairArgs>& pairs, int p1h, int p2h, int paths,
                       const BatchTiles& t, unsigned char* scratch, unsigned char* d_desc, BatchPlan& out);
// Opts the persistent kernel into the plan's dynamic shared memory.
cudaError_t batch_configure(const BatchPlan& plan);
// Zeroes the control words and launches the persistent kernel (grid blocks);
// batch_configure must have run for a plan of at least this shared memory.
// trace: null, or 4 words per queue item (taken, dependency met, ended, smid << 32 | pair * 16 + pass)
cudaError_t batch_launch(const BatchPlan& plan, unsigned char* d_desc, unsigned long long wait_ns, int grid,
                         cudaStream_t st, unsigned long long* trace = nullptr);

// Differentiable soft-argmin SGM (kernels_soft.cu).
struct SoftLaunch {
    int f64;
    const void* cost;
    void* part;  // scratch: one volume per direction (forward L, backward dC contributions)
    void* S;
    void* dS;
    void* dcost;
    void* codes;
    void* kstar;
    void* ckpt;
    const long long* ckpt_off;
    void* dhat;
    void* stats;
    const void* g;
    void* dpen;
    void* dpen_part;
    int W, H, D, paths, ck, record;
    double p1, p2, tau;
};
cudaError_t launch_soft_forward(const SoftLaunch& a, cudaStream_t st, Timer* tm);
cudaError_t launch_soft_backward(const SoftLaunch& a, cudaStream_t st, Timer* tm);

}  // namespace tdv
