/*
 * tdv_stereo.h -- C ABI of the B200 (sm_100a) dense-stereo hot path:
 * matching-cost DSI -> SGM / DP aggregation -> WTA disparity reduction.
 *
 * Every entry point takes plain device pointers and sizes, runs asynchronously
 * on the caller's CUDA stream (NULL = legacy default stream) and returns a
 * tdv_status; nothing is thrown across the ABI.  The reference (ThunderVision's
 * LibThunderVision) reaches the same stages through free C++ functions with no
 * extern "C"; each declaration below names the reference function it replaces
 * (paths relative to the ThunderVision root; tdvision/ =
 * LibThunderVision/src/tdvision/).
 *
 * Conventions
 *   - Images are single-channel, row-major, device memory: u8 or f32, with a
 *     row pitch in elements and an intensity scale (intensity = value*scale;
 *     scale 1/255 is the reference's [0,1] domain, tdvision/misc.cpp:31-32).
 *   - Cost / aggregation volumes ("DSI") keep the disparity axis contiguous.
 *     TDV_LAYOUT_REF_WHD is the reference layout, offset ((x*H)+y)*D+d with a
 *     row pitch of D elements (tdvision/dsimem.cpp:34-35, dsimemutil.h:6);
 *     TDV_LAYOUT_HWD is ((y*W)+x)*D+d.
 *   - Cells with x-d < 0 hold +INF (tdvision/birchfieldcost.cu:52).
 *   - Disparity outputs are W*H arrays: uint16 disparity (0xFFFF = rejected by
 *     the left-right check) and/or float d/D, the reference's output format
 *     (tdvision/wtacpu.cpp:35-36).
 */
#ifndef TDV_STEREO_H
#define TDV_STEREO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TDV_ABI_VERSION 1

typedef struct tdv_ctx tdv_ctx;
typedef void* tdv_stream; /* a cudaStream_t */

/* Replaces the reference's exception convention (CUException thrown by
 * CUerrExp, tdvision/cuerr.hpp:73-78, cuerr.cpp:6-15). */
typedef enum {
    TDV_OK = 0,
    TDV_ERR_INVALID_ARG = 1,
    TDV_ERR_UNSUPPORTED = 2,
    TDV_ERR_OOM = 3,
    TDV_ERR_CUDA = 4,
    TDV_ERR_TIMEOUT = 5,
    TDV_ERR_BAD_WORK = 6
} tdv_status;

typedef enum { TDV_LAYOUT_REF_WHD = 0, TDV_LAYOUT_HWD = 1 } tdv_layout;
typedef enum { TDV_F32 = 0, TDV_U16 = 1, TDV_U8 = 2, TDV_F64 = 3 } tdv_dtype;

typedef struct {
    const void* ptr;  /* device */
    int32_t width, height;
    int32_t pitch;    /* elements between rows, >= width */
    int32_t dtype;    /* TDV_U8 or TDV_F32 */
    float scale;      /* intensity = value * scale */
} tdv_image;

typedef struct {
    void* ptr;        /* device, dense, no padding between pixels */
    int32_t width, height, depth;
    int32_t layout;   /* tdv_layout */
    int32_t dtype;    /* TDV_F32; cost DSIs may be TDV_U16 (BT of TDV_U8 images at
                         scale 1, in half-units: value = 2 * cost, +INF = 0xFFFF,
                         exact) for tdv_cost, tdv_sgm's cost, tdv_wta and
                         tdv_dp_scanline; the soft-SGM calls also take TDV_F64 */
} tdv_volume;

typedef struct {
    uint16_t* disp;       /* W*H disparity, may be NULL */
    float* disp_norm;     /* W*H d/D (reference format), may be NULL */
    uint16_t* disp_right; /* W*H right-view disparity, may be NULL */
    int32_t lr_threshold; /* < 0: no left-right check; else reject |dL-dR|>thr */
} tdv_disparity;

/* ---- matching cost --------------------------------------------------- */
typedef enum { TDV_COST_BT = 0, TDV_COST_SSD = 1, TDV_COST_NCC = 2 } tdv_cost_kind;

typedef struct {
    int32_t kind;   /* tdv_cost_kind */
    int32_t radius; /* SSD/NCC window radius: SSD 3 = the reference's 7x7
                       (tdvision/ssd.cu:11-13), NCC 1 = its 3x3
                       (tdvision/crosscorrelation.cu:17-18); ignored for BT */
} tdv_cost_params;

/* Fills the cost DSI `out` (F32, either layout; or U16 for BT of u8 images
 * at scale 1, else TDV_ERR_UNSUPPORTED) from a rectified pair.
 * Replaces BirchfieldCostRun (tdvision/birchfieldcost.cu:194-212),
 * SSDDevRun (tdvision/ssd.cu:79-114) and CrossCorrelationDevRun
 * (tdvision/crosscorrelation.cu:53-76), i.e. the updateImpl of
 * AbstractMatchingCost (tdvision/matchingcost.hpp:48-49). */
tdv_status tdv_cost(tdv_ctx* ctx, const tdv_image* left, const tdv_image* right,
                    const tdv_cost_params* params, tdv_volume* out, tdv_stream stream);

/* The cost of a pre-filtered pair, DevStereoMatcher's default chain
 * (tdvision/devstereomatcher.cpp:13-48: MedianFilterCPU on both inputs, then
 * the matching cost): `filter` (tdv_filter_kind, declared with tdv_prefilter)
 * is applied to both images, value * scale, then the cost is taken over the
 * filtered images exactly as tdv_cost takes it.  For TDV_FILTER_GAUSS5 with
 * BT, or SSD / NCC of radius 1..4, the Gaussian runs inside the cost
 * kernel's shared-memory staging and the filtered images are never stored;
 * other cases filter into context scratch first.  Bit-identical to
 * tdv_prefilter on both images followed by tdv_cost.  `left_filtered` (F32,
 * the DSI's width x height, dense; NULL to skip) receives the filtered left
 * image, the guide tdv_sgm's adjusted P2 reads (DSIMem::leftOrigin is the
 * filtered left image, tdvision/matchingcost.cpp:30-33). */
tdv_status tdv_cost_filtered(tdv_ctx* ctx, const tdv_image* left, const tdv_image* right,
                             const tdv_cost_params* params, int32_t filter, tdv_volume* out,
                             float* left_filtered, tdv_stream stream);

/* ---- semi-global aggregation ----------------------------------------- */
typedef enum {
    TDV_SEM_STANDARD = 0, /* S += C at path starts, previous = C, full min over d */
    TDV_SEM_REF_CPU = 1,  /* tdvision/semiglobalcpu.cpp:56-126 as written */
    TDV_SEM_REF_GPU = 2   /* tdvision/semiglobal.cu:283-466 without its race */
} tdv_sgm_semantics;
typedef enum { TDV_TABLE_FULL = 0, TDV_TABLE_REF = 1 } tdv_path_table;
typedef enum { TDV_P2_CONST = 0, TDV_P2_ADJUST = 1 } tdv_p2_mode;

typedef struct {
    float p1, p2;      /* penalties (reference: 30/255, 150/255,
                          tdvision/semiglobalcpu.cpp:36-37) */
    int32_t p2_mode;   /* tdv_p2_mode: ADJUST = P2/|I(p)-I(p-r)| */
    int32_t paths;     /* 8, or 4 (horizontal + vertical) */
    int32_t table;     /* tdv_path_table: REF = the reference's SGPaths as built
                          by tdvision/semiglobal.cu:57-230 */
    int32_t semantics; /* tdv_sgm_semantics */
} tdv_sgm_params;

/* Aggregates a cost DSI and reduces it to disparities (fused WTA, optional
 * left-right check).  `guide` is the intensity image for P2_ADJUST (may be
 * NULL otherwise).  `aggreg` (optional, F32, same layout as `cost`) receives
 * the aggregated volume.  Replaces SemiGlobalDevRun
 * (tdvision/semiglobal.cu:474-521) and SemiGlobalCPU::updateImpl
 * (tdvision/semiglobalcpu.cpp:173-230). */
tdv_status tdv_sgm(tdv_ctx* ctx, const tdv_volume* cost, const tdv_image* guide,
                   const tdv_sgm_params* params, tdv_volume* aggreg, tdv_disparity* out,
                   tdv_stream stream);

/* Winner-take-all over a DSI, lowest d on ties.  Replaces WTARunDev
 * (tdvision/wta.cu:90-100) and WTACPU::wta (tdvision/wtacpu.cpp:14-39). */
tdv_status tdv_wta(tdv_ctx* ctx, const tdv_volume* vol, tdv_disparity* out, tdv_stream stream);

/* Dynamic-programming scanline matcher over a cost DSI.  Replaces
 * DynamicProgDevRun (tdvision/dynamicprog.cu:106-122). */
tdv_status tdv_dp_scanline(tdv_ctx* ctx, const tdv_volume* cost, tdv_disparity* out,
                           tdv_stream stream);

/* SSD window + WTA fused, no DSI.  Replaces FastWTADevRun
 * (tdvision/fastwta.cu:57-83). */
tdv_status tdv_fast_wta(tdv_ctx* ctx, const tdv_image* left, const tdv_image* right,
                        int32_t max_disp, int32_t radius, tdv_disparity* out, tdv_stream stream);

/* Birchfield-Tomasi cost recomputed inside the aggregation, no cost DSI:
 * the role of SemiGlobalLabDevRun (tdvision/semiglobal_lab.cu:232-282) with
 * the reference's cost and recurrence.  Integer-domain inputs (u8, scale 1,
 * P1/P2 multiples of 1/2, P2_CONST, D <= 256; any semantics and table whose
 * 16-bit ranges hold) take the fused 16-bit path; anything else runs
 * tdv_cost + tdv_sgm on context scratch. */
tdv_status tdv_stereo_sgm(tdv_ctx* ctx, const tdv_image* left, const tdv_image* right,
                          int32_t max_disp, const tdv_sgm_params* params, tdv_disparity* out,
                          tdv_stream stream);

/* tdv_stereo_sgm's fused path over n frame pairs of one size (left[i],
 * right[i] -> out[i]), for a frame stream: the frames alternate between two
 * lanes, each with its own planes, aggregation volumes and streams, so that
 * one frame's DRAM-bound passes run while the other lane's last pass (WTA and
 * left-right check, bound by its instruction stream) finishes.  The call
 * orders everything after the work already queued on `stream` and before the
 * work queued on it afterwards; the outputs must not overlap one another.
 * Maps are identical to n tdv_stereo_sgm calls.  Inputs outside the fused
 * path return TDV_ERR_UNSUPPORTED.  The second lane's scratch (about as much
 * as the first's) is allocated on the first call with n > 1.  No reference
 * counterpart: the reference matches one pair per pipeline update
 * (tdvision/devstereomatcher.cpp:36-48). */
tdv_status tdv_stereo_sgm_frames(tdv_ctx* ctx, int32_t n, const tdv_image* left, const tdv_image* right,
                                 int32_t max_disp, const tdv_sgm_params* params, tdv_disparity* out,
                                 tdv_stream stream);

/* Allocation-free variant of tdv_stereo_sgm's fused integer-domain path, for
 * callers that cannot call cudaMalloc while they run (a capture or control
 * loop with a device-memory budget fixed at start-up, a plugin whose host owns
 * every allocation, a real-time frame loop that must not stall on an
 * allocation).  It has no counterpart in the reference.  All scratch comes
 * from one 64 MiB static __device__ array held by every GPU that loads this
 * library until the process exits.  A pair needs the BT planes,
 * 16*(W + 9*ceil(W/8)) bytes per row (about 34 B per pixel), plus the
 * aggregation volume, 128 B per pixel for D <= 64, 256 B for D <= 128 and
 * 512 B for D <= 256, each rounded up to 256 bytes, plus 256 bytes; pairs
 * that do not fit, and inputs outside the fused path, are rejected with
 * TDV_ERR_UNSUPPORTED, malformed arguments (non-finite penalties, values
 * outside the enums, sizes that differ) with TDV_ERR_INVALID_ARG.  The first
 * call on a device, and the first after a device reset or in another context
 * there, resolves the array's address; make it before any stream capture (a
 * capturing call cannot and returns TDV_ERR_INVALID_ARG).  Calls share the
 * array: calls whose GPU work overlaps race.  If a bounded wait inside the
 * kernels runs out, every pixel of the requested outputs is marked invalid
 * (0xFFFF, -1.0f). */
tdv_status tdv_stereo_sgm_static(const tdv_image* left, const tdv_image* right, int32_t max_disp,
                                 const tdv_sgm_params* params, tdv_disparity* out, tdv_stream stream);

/* ---- batched pairs: one persistent launch (no reference counterpart) ----
 * The reference matches one pair per pipeline update
 * (tdvision/devstereomatcher.cpp:36-48 chains the cost and optimizer stages
 * of one frame); these calls run the fused integer-domain path of
 * tdv_stereo_sgm over many pairs of uneven size and disparity range in one
 * persistent kernel fed by a device work queue, with results bit-identical
 * to per-pair tdv_stereo_sgm calls. */
typedef struct {
    tdv_image left, right; /* TDV_U8, scale 1, device memory, equal sizes */
    int32_t max_disp;      /* 1..256 */
    tdv_disparity out;     /* as for tdv_stereo_sgm */
} tdv_batch_pair;

typedef enum { TDV_BATCH_ORDER_LONGEST_FIRST = 0, TDV_BATCH_ORDER_INPUT = 1 } tdv_batch_order;

/* Tile shapes of the persistent kernel. */
typedef struct {
    int32_t lines_per_cta;   /* vertical/diagonal passes: path lines per block, 1..24 */
    int32_t rows_per_cta;    /* horizontal passes: image rows per block, 1..25 (12 when split) */
    int32_t split_disparity; /* horizontal passes, D > 64: 1 = two warps share a row's
                                disparity range, 0 = one warp per row */
    int32_t order;           /* tdv_batch_order: pairs inside each pass of the queue */
    int32_t ctas_per_sm;     /* 1: one 25-warp block per SM; 2: two 13-warp blocks per SM,
                                each taking its own work items (lines and rows per block
                                then at most 12) */
} tdv_batch_tiles;

typedef struct tdv_batch tdv_batch;

/* Plans a batch: validates every pair (integer-domain fused path only:
 * P1/P2 multiples of 1/2, P2 <= 1280, STANDARD, FULL, P2_CONST), allocates
 * the planes and aggregation volumes of all pairs and the device work queue
 * from the context's allocator, and uploads the queue built with the default
 * tiles.  The pair pointers are fixed at creation (a video loop rewrites the
 * same input buffers and relaunches). */
tdv_status tdv_batch_create(tdv_ctx* ctx, const tdv_batch_pair* pairs, int32_t n_pairs,
                            const tdv_sgm_params* params, tdv_batch** out);
void tdv_batch_destroy(tdv_batch* batch);
tdv_status tdv_batch_set_tiles(tdv_batch* batch, const tdv_batch_tiles* tiles);
tdv_status tdv_batch_get_tiles(const tdv_batch* batch, tdv_batch_tiles* tiles);
/* Times candidate tile shapes on this batch (each run `reps` times on
 * `stream`, device time by CUDA events), keeps the fastest and returns it
 * with its milliseconds per run. */
tdv_status tdv_batch_autotune(tdv_batch* batch, int32_t reps, tdv_stream stream,
                              tdv_batch_tiles* chosen, double* best_ms);
/* One run: zero the queue's control words, one persistent launch. */
tdv_status tdv_batch_run(tdv_batch* batch, tdv_stream stream);
/* The same run through a CUDA graph, captured on first use (and again after
 * the tiles change) and replayed on `stream`. */
tdv_status tdv_batch_graph_launch(tdv_batch* batch, tdv_stream stream);
/* Synchronises `stream` and returns the device status of the last run:
 * TDV_ERR_TIMEOUT (a bounded wait ran out), TDV_ERR_BAD_WORK (a work item out
 * of range), else TDV_OK. */
tdv_status tdv_batch_status(tdv_batch* batch, tdv_stream stream);
/* Bounded-wait limit for the kernel's dependency waits (default 2 s). */
tdv_status tdv_batch_set_wait_limit(tdv_batch* batch, double seconds);
/* Diagnostic trace of the runs that follow: `trace` (device memory, at least
 * 4 * n_items 64-bit words, or NULL to stop) receives per queue item the
 * global timer (ns) when a block took it, when its dependency was met and
 * when it ended, and smid << 32 | (pair * 16 + pass).  Where the persistent kernel
 * waits and where it idles at the end can be read from it. */
tdv_status tdv_batch_set_trace(tdv_batch* batch, unsigned long long* trace, int64_t capacity_items);
/* The device work queue (n_items entries of item_bytes: int32 pair*16+pass,
 * int32 block), pass-major, and the per-pass item counts; for inspection and
 * for tests that plant faults in the queue. */
tdv_status tdv_batch_work_queue(tdv_batch* batch, void** items, int32_t* n_items, int32_t* item_bytes);

/* ---- differentiable soft-argmin SGM (no reference counterpart) --------- */
typedef struct {
    double p1, p2;      /* penalties, constant P2 (double so FP64 runs keep them exact) */
    int32_t paths;      /* 8 or 4 */
    double tau;         /* softmin temperature, > 0 */
    int32_t checkpoint; /* 0: the tape keeps 2-bit choice codes of every cell;
                           k in [1,32]: it keeps L every k steps of each path
                           and the adjoint recomputes one k-step segment at a
                           time */
} tdv_soft_params;

/* Bytes of the tape tdv_soft_sgm_forward records for the adjoint. */
size_t tdv_soft_sgm_tape_bytes(int32_t width, int32_t height, int32_t depth, int32_t dtype,
                               const tdv_soft_params* params);

/* Expected disparity dhat = sum_d d*softmax(-S/tau) of the STANDARD 4/8-path
 * aggregation S of `cost` (HWD layout, TDV_F32 or TDV_F64); dhat is W*H of
 * the cost's dtype.  With `tape` (tdv_soft_sgm_tape_bytes bytes, device) the
 * call records what tdv_soft_sgm_backward needs; with tape = NULL it only
 * evaluates. */
tdv_status tdv_soft_sgm_forward(tdv_ctx* ctx, const tdv_volume* cost, const tdv_soft_params* params,
                                void* dhat, void* tape, size_t tape_bytes, tdv_stream stream);

/* Adjoint of tdv_soft_sgm_forward: given g = dLoss/d(dhat) (W*H), writes
 * dLoss/dcost into `dcost` (same shape/dtype as the cost) and
 * (dLoss/dP1, dLoss/dP2) into dpen[0..1] (device, cost dtype). */
tdv_status tdv_soft_sgm_backward(tdv_ctx* ctx, const tdv_volume* cost, const tdv_soft_params* params,
                                 const void* tape, size_t tape_bytes, const void* g_dhat,
                                 tdv_volume* dcost, void* dpen, tdv_stream stream);

/* ---- image stages either side of the path ------------------------------
 * The steps LibThunderVision runs before the cost (input conversion,
 * rectification remap, pre-filter) and after the disparity reduction
 * (morphological clean-up, sub-pixel refinement, reprojection to 3D and the
 * PLY mesh file), as device kernels on caller-owned buffers. */

/* A 2-D array of pixels with interleaved channels. */
typedef struct {
    void* ptr;           /* device */
    int32_t width, height;
    int32_t pitch_bytes; /* bytes between rows, >= width * channels * element size */
    int32_t dtype;       /* TDV_U8, TDV_U16 or TDV_F32 */
    int32_t channels;    /* 1 or 3 */
} tdv_raster;

/* Grey conversion of an 8-bit 3-channel image into F32: each channel scaled
 * by 1/255 (in double, rounded to float), then 0.299*c0 + 0.587*c1 + 0.114*c2
 * with channel 0 weighted as red whatever the capture order, as the reference
 * converts its BGR frames (tdvision/misc.cpp:29-32). */
tdv_status tdv_to_gray(tdv_ctx* ctx, const tdv_raster* color, float* gray, tdv_stream stream);

/* Rectification maps of one camera: for each pixel (j, i) of the rectified
 * width x height image, the source position after R, the new camera P and
 * the Brown-Conrady distortion of K, dist = (k1, k2, p1, p2, k3, k4, k5, k6)
 * (zeros for unused terms): (X, Y, W) = inv(P[:, :3] R) (j, i, 1) (inverse by
 * cofactors), x = X/W, y = Y/W, r2 = x^2 + y^2,
 * kr = (1 + ((k3 r2 + k2) r2 + k1) r2) / (1 + ((k6 r2 + k5) r2 + k4) r2),
 * mapx = fx (x kr + 2 p1 x y + p2 (r2 + 2 x^2)) + cx,
 * mapy = fy (y kr + p1 (r2 + 2 y^2) + 2 p2 x y) + cy, in double, stored as
 * float.  Replaces the cvInitUndistortRectifyMap calls of RectificationCV
 * (tdvision/rectificationcv.cpp:114-117, 152-155); K, R, P row-major 3x3
 * (P's first three columns). */
tdv_status tdv_rectify_maps(tdv_ctx* ctx, const double* K, const double* dist, const double* R,
                            const double* P, int32_t width, int32_t height, float* mapx, float* mapy,
                            tdv_stream stream);

/* Rectification remap: dst(x, y) = src sampled bilinearly at (mapx, mapy)
 * (float maps of dst's size, dense rows), coordinates rounded to 1/32 pixel,
 * taps outside src read 0; U8 sources use 15-bit fixed-point weights with
 * rounding, F32 sources float weights.  Replaces the per-frame cvRemap of
 * RectificationCV::update (tdvision/rectificationcv.cpp:298-310); src and dst
 * have the same dtype and channel count. */
tdv_status tdv_remap(tdv_ctx* ctx, const tdv_raster* src, const float* mapx, const float* mapy,
                     tdv_raster* dst, tdv_stream stream);

typedef enum {
    TDV_FILTER_GAUSS5 = 0,  /* separable [1 4 6 4 1]/16, replicated borders: the 5x5 Gaussian
                               DevStereoMatcher applies by default (MedianFilterCPU =
                               cvSmooth(CV_GAUSSIAN, 5), tdvision/medianfiltercpu.cpp:15,
                               devstereomatcher.cpp:11,22-29) */
    TDV_FILTER_MEDIAN7 = 1  /* 7x7 median, replicated borders: the median the reference's
                               device filter was written for (tdvision/medianfilter.cu:37-57;
                               its launcher runs a placeholder instead, :75-76) */
} tdv_filter_kind;

/* Pre-filter of one image before the cost: `out` is F32, width x height,
 * dense rows, holding the filtered intensities (value * scale). */
tdv_status tdv_prefilter(tdv_ctx* ctx, const tdv_image* in, int32_t kind, float* out, tdv_stream stream);

typedef enum {
    TDV_POST_OPEN7 = 0,   /* 7x7 minimum then 7x7 maximum, windows clipped at the borders:
                             Dilate's cvErode + cvDilate with 3 iterations of the default 3x3
                             element (tdvision/dilate.cpp:18-19), run after the matcher in
                             Reconstruction (tdvision/reconstruction.cpp:30-31) */
    TDV_POST_MEDIAN3 = 1  /* 3x3 median, replicated borders */
} tdv_post_kind;

/* Post-filter of a 1-channel disparity map (F32 or U16); in and out have the
 * same size and dtype and must not overlap. */
tdv_status tdv_postfilter(tdv_ctx* ctx, const tdv_raster* in, int32_t kind, tdv_raster* out,
                          tdv_stream stream);

/* Sub-pixel refinement: for each pixel with 0 < d < D-1 and a convex
 * neighbourhood, d + (S(d-1) - S(d+1)) / (2 (S(d-1) - 2 S(d) + S(d+1))) from the
 * aggregated volume S (F32, HWD, as tdv_sgm writes it); other pixels keep d,
 * invalid ones (0xFFFF) give -1.  `out` is F32 width x height. */
tdv_status tdv_subpixel(tdv_ctx* ctx, const tdv_volume* S, const uint16_t* disp, float* out,
                        tdv_stream stream);

typedef enum {
    TDV_REPROJECT_DIRECT = 0, /* (x, H - y, d * zscale): DirectReprojector::reproject
                                 (tdvision/directreprojector.hpp:17-20) */
    TDV_REPROJECT_Q = 1       /* Q * (x, H - y, d, 1), divided by w (0 when |w| <= FLT_EPSILON),
                                 then z * 24: CVReprojector::reproject
                                 (tdvision/cvreprojector.cpp:45-60) */
} tdv_reproject_mode;

typedef struct {
    int32_t mode;  /* tdv_reproject_mode */
    float zscale;  /* DIRECT */
    float q[16];   /* Q, row-major (cvStereoRectify's reprojection matrix) */
} tdv_reproject_params;

/* Reprojection of a disparity map (F32, 1 channel: the values the matcher's
 * float output holds) to one vertex per pixel, row-major, 3 floats each, and
 * the pixel's color (U8, 3 channels, may be NULL) to 3 floats in [0, 1]
 * (channel order kept), as GLReprojection::updateMesh fills the grid mesh
 * (tdvision/glreprojection.cpp:30-55), into device buffers. */
tdv_status tdv_reproject(tdv_ctx* ctx, const tdv_raster* disp, const tdv_raster* color,
                         const tdv_reproject_params* params, float* vertices, float* colors,
                         tdv_stream stream);

/* Writes the grid mesh (host vertices and colors as tdv_reproject lays them
 * out) as the reference's ASCII PLY: a vertex per pixel "x y z r g b" with the
 * colors times 255 truncated, then a quad "4 a b c d" per grid cell
 * (tdvision/plymeshexporter.cpp:8-76).  colors may be NULL (0 0 0). */
tdv_status tdv_write_ply(const char* path, const float* vertices, const float* colors, int32_t width,
                         int32_t height);

/* ---- context ---------------------------------------------------------- */
typedef void* (*tdv_alloc_fn)(size_t bytes, void* user);
typedef void (*tdv_free_fn)(void* ptr, void* user);

/* Creates a context bound to `device`; no CUDA call is made until first use.
 * A context owns scratch (aggregation volumes, path tables); use one per host
 * thread.  Replaces the per-stage scratch of SemiGlobalDev / DynamicProgDev
 * (tdvision/semiglobaldev.hpp:19-21, dynamicprogdev.hpp:14-15). */
tdv_status tdv_ctx_create(int32_t device, tdv_ctx** out);
void tdv_ctx_destroy(tdv_ctx* ctx);
/* Replaces the device allocator for scratch (default cudaMalloc/cudaFree). */
tdv_status tdv_ctx_set_allocator(tdv_ctx* ctx, tdv_alloc_fn alloc, tdv_free_fn release,
                                 void* user);
/* Pre-sizes the scratch of tdv_stereo_sgm (the fused path: planes, both
 * 16-bit aggregation volumes, the row scratch) for pairs up to W x H x D, so
 * later calls of it do not allocate.  The general path sizes its own scratch
 * on first use, once per size: tdv_sgm without a caller aggregation volume
 * (W x H x D floats, the path schedule, the deferred costs of repeated
 * walks), tdv_dp_scanline (W x H x D choice bytes), the filter-then-cost
 * case of tdv_cost_filtered (both filtered images).  A caller that must not
 * allocate later makes one call of each kind first, or passes its own
 * volumes. */
tdv_status tdv_ctx_reserve(tdv_ctx* ctx, int32_t width, int32_t height, int32_t max_disp);
const char* tdv_last_error_string(const tdv_ctx* ctx);
/* Synchronises `stream` and returns the error status kernels of this
 * context recorded on the device (TDV_ERR_TIMEOUT when a bounded wait inside
 * a kernel ran out), clearing it; TDV_OK if none. */
tdv_status tdv_ctx_device_status(tdv_ctx* ctx, tdv_stream stream);
/* Per-kernel timing: when enabled, every kernel a call launches is bracketed
 * by CUDA events on the call's stream; tdv_ctx_timings then returns (after the
 * stream has been synchronised) the device milliseconds of each launch of the
 * most recent call and tdv_ctx_timing_name its kernel name.  This replaces the
 * reference's CudaBenchmarker around each stage update
 * (tdvision/benchmark.cpp:7-31, matchingcost.cpp:35-42).  While timing is on,
 * work a call would run concurrently on two streams (the fused 8-path pass
 * chains) runs in sequence on the call's stream, so each kernel is timed
 * alone. */
tdv_status tdv_ctx_enable_timing(tdv_ctx* ctx, int32_t enable);
int32_t tdv_ctx_timings(tdv_ctx* ctx, float* ms_out, int32_t max_entries);
const char* tdv_ctx_timing_name(const tdv_ctx* ctx, int32_t index);
const char* tdv_status_string(tdv_status status);
int32_t tdv_version(void);
/* Bytes of a dense W x H x D volume of `dtype`. */
size_t tdv_volume_bytes(int32_t width, int32_t height, int32_t depth, int32_t dtype);

#ifdef __cplusplus
}
#endif

#endif /* TDV_STEREO_H */
