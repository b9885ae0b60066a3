// tdv_stages.hpp -- C++ stage classes over the C ABI (tdv_stereo.h), named
// and shaped like LibThunderVision's stage plugins so that host code written
// against the reference's stages reads the same:
//
//   reference (tdvision/)                      here (namespace tdv_b200)
//   MatchingCost::updateImpl(L, R, DSIMem)      MatchingCost::update(L, R, dsi)
//     (matchingcost.hpp:48-49)
//   BirchfieldCostDev (birchfieldcostdev.hpp)   BirchfieldCostDev
//   SSDDev (ssddev.hpp, 7x7 window)             SSDDev (radius 3 by default)
//   CrossCorrelationDev (crosscorrelationdev.hpp, 3x3)  CrossCorrelationDev
//   Optimizer::updateImpl(DSIMem, FloatImage)   Optimizer::update(dsi, out)
//     (optimizer.hpp:46)
//   SemiGlobalDev (semiglobaldev.hpp)           SemiGlobalDev  (REF_GPU semantics)
//   SemiGlobalCPU (semiglobalcpu.hpp)           SemiGlobalCPU  (REF_CPU semantics)
//   WTADev / WTACPU (wtadev.hpp, wtacpu.hpp)    WTADev
//   DynamicProgDev (dynamicprogdev.hpp)         DynamicProgDev
//   FastWTAMatcher (fastwtamatcher.hpp)         FastWTAMatcher
//   SemiGlobalLabMatcher (semigloballabmatcher.hpp)  SemiGlobalLabMatcher
//   misc::create32FGray (misc.cpp:18-32)        create32FGray
//   RectificationCV, calibrated path            Rectifier (maps once, remap per frame)
//     (rectificationcv.cpp:114-117, 298-310)
//   MedianFilterCPU (5x5 Gaussian, medianfiltercpu.cpp:15)  MedianFilterCPU
//   MedianFilterDev (7x7 median, medianfilter.cu:37-57)     MedianFilterDev
//   Dilate (dilate.cpp:11-22)                   Dilate
//   DirectReprojector / CVReprojector           DirectReprojector / CVReprojector
//     (directreprojector.hpp, cvreprojector.cpp:45-60)
//   PLYMeshExporter::exportMesh (plymeshexporter.cpp)  PLYMeshExporter
//
// The reference's stages pull their inputs from pipes and run on worker
// threads (workunitprocess.cpp); that runtime is not part of this path, so
// each stage here takes its buffers as arguments and runs on a CUDA stream.
// Errors throw CUException, as the reference's stages do (cuerr.hpp:73-78).
// Everything is device memory; nothing runs on the host.
#ifndef TDV_STAGES_HPP
#define TDV_STAGES_HPP

#include <stdexcept>
#include <string>

#include "tdv_stereo.h"

namespace tdv_b200 {

class CUException : public std::runtime_error {
public:
    CUException(tdv_status status, const std::string& what) : std::runtime_error(what), m_status(status) {}
    tdv_status status() const { return m_status; }

private:
    tdv_status m_status;
};

inline void check(tdv_ctx* ctx, tdv_status st) {
    if (st != TDV_OK)
        throw CUException(st, std::string(tdv_status_string(st)) + ": " + tdv_last_error_string(ctx));
}

// A float image in device memory, intensities in [0,1] (the reference's
// FloatImage device buffer, floatimage.hpp; misc.cpp:31-32).
struct FloatImage {
    const float* devMem = nullptr;
    int width = 0, height = 0;
    tdv_image abi(float scale = 1.0f) const {
        tdv_image im;
        im.ptr = devMem;
        im.width = width;
        im.height = height;
        im.pitch = width;
        im.dtype = TDV_F32;
        im.scale = scale;
        return im;
    }
};

// A u8 image in device memory (the fused matchers' input).
struct ByteImage {
    const unsigned char* devMem = nullptr;
    int width = 0, height = 0, pitch = 0;
    tdv_image abi() const {
        tdv_image im;
        im.ptr = devMem;
        im.width = width;
        im.height = height;
        im.pitch = pitch > 0 ? pitch : width;
        im.dtype = TDV_U8;
        im.scale = 1.0f;
        return im;
    }
};

// A cost / aggregation volume in the reference's layout ((x*H)+y)*D+d
// (DSIMem, dsimem.cpp:34-35) or HWD, plus the left image it was computed
// from (DSIMem::leftOrigin, used by P2_ADJUST).
struct DSIMem {
    float* devMem = nullptr;
    int width = 0, height = 0, depth = 0;
    int layout = TDV_LAYOUT_REF_WHD;
    FloatImage leftOrigin;
    tdv_volume abi() const {
        tdv_volume v;
        v.ptr = devMem;
        v.width = width;
        v.height = height;
        v.depth = depth;
        v.layout = layout;
        v.dtype = TDV_F32;
        return v;
    }
};

// Disparity outputs (any may be null): u16 disparities, d/D floats (the
// reference's output image, wtacpu.cpp:35-36), right-view disparities.
struct Disparity {
    unsigned short* disp = nullptr;
    float* dispNorm = nullptr;
    unsigned short* dispRight = nullptr;
    int lrThreshold = -1;
    tdv_disparity abi() const {
        tdv_disparity o;
        o.disp = disp;
        o.disp_norm = dispNorm;
        o.disp_right = dispRight;
        o.lr_threshold = lrThreshold;
        return o;
    }
};

// Owns a tdv_ctx (scratch, schedules) on one device.
class Context {
public:
    explicit Context(int device = 0) { check(nullptr, tdv_ctx_create(device, &m_ctx)); }
    ~Context() { tdv_ctx_destroy(m_ctx); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    tdv_ctx* get() const { return m_ctx; }
    void reserve(int w, int h, int d) { check(m_ctx, tdv_ctx_reserve(m_ctx, w, h, d)); }
    void deviceStatus(tdv_stream s = nullptr) { check(m_ctx, tdv_ctx_device_status(m_ctx, s)); }

private:
    tdv_ctx* m_ctx = nullptr;
};

// ---- matching cost stages (AbstractMatchingCost::updateImpl) -------------
class MatchingCost {
public:
    MatchingCost(Context& ctx, int disparityMax, tdv_cost_kind kind, int radius)
        : m_ctx(ctx), m_disparityMax(disparityMax) {
        m_params.kind = kind;
        m_params.radius = radius;
    }
    virtual ~MatchingCost() {}
    int disparityMax() const { return m_disparityMax; }
    // fills `dsi` (W x H x disparityMax, either layout) from the pair
    void update(const FloatImage& left, const FloatImage& right, DSIMem& dsi, tdv_stream s = nullptr) {
        tdv_image l = left.abi(), r = right.abi();
        tdv_volume v = dsi.abi();
        check(m_ctx.get(), tdv_cost(m_ctx.get(), &l, &r, &m_params, &v, s));
        dsi.leftOrigin = left;
    }
    // DevStereoMatcher's default chain (devstereomatcher.cpp:22-29): both
    // images pass `filter` (the 5x5 Gaussian fused into the cost kernel)
    // before the cost; the filtered left image goes to `filteredLeft`
    // (dsi.width x dsi.height floats) and becomes dsi.leftOrigin, the guide
    // of an adjusted P2
    void update(const FloatImage& left, const FloatImage& right, DSIMem& dsi, float* filteredLeft,
                tdv_filter_kind filter = TDV_FILTER_GAUSS5, tdv_stream s = nullptr) {
        tdv_image l = left.abi(), r = right.abi();
        tdv_volume v = dsi.abi();
        check(m_ctx.get(), tdv_cost_filtered(m_ctx.get(), &l, &r, &m_params, filter, &v, filteredLeft, s));
        dsi.leftOrigin = FloatImage{filteredLeft, dsi.width, dsi.height};
    }

protected:
    Context& m_ctx;
    int m_disparityMax;
    tdv_cost_params m_params;
};

class BirchfieldCostDev : public MatchingCost {
public:
    BirchfieldCostDev(Context& ctx, int disparityMax) : MatchingCost(ctx, disparityMax, TDV_COST_BT, 0) {}
};

class SSDDev : public MatchingCost {
public:
    SSDDev(Context& ctx, int disparityMax, int radius = 3) : MatchingCost(ctx, disparityMax, TDV_COST_SSD, radius) {}
};

class CrossCorrelationDev : public MatchingCost {
public:
    CrossCorrelationDev(Context& ctx, int disparityMax, int radius = 1)
        : MatchingCost(ctx, disparityMax, TDV_COST_NCC, radius) {}
};

// ---- optimizer stages (AbstractOptimizer::updateImpl) --------------------
class Optimizer {
public:
    explicit Optimizer(Context& ctx) : m_ctx(ctx) {}
    virtual ~Optimizer() {}
    virtual void update(const DSIMem& dsi, Disparity& out, tdv_stream s = nullptr) = 0;

protected:
    Context& m_ctx;
};

// SGM + WTA; the defaults are the reference's (semiglobalcpu.cpp:36-37:
// P1 = 30/255, P2 = 150/255 divided by the intensity step, its path table).
class SemiGlobalOptimizer : public Optimizer {
public:
    SemiGlobalOptimizer(Context& ctx, tdv_sgm_semantics sem) : Optimizer(ctx) {
        m_params.p1 = 30.0f / 255.0f;
        m_params.p2 = 150.0f / 255.0f;
        m_params.p2_mode = TDV_P2_ADJUST;
        m_params.paths = 8;
        m_params.table = TDV_TABLE_REF;
        m_params.semantics = sem;
    }
    tdv_sgm_params& params() { return m_params; }
    // aggregated volume (optional, same shape and layout as the cost)
    void aggregation(DSIMem* aggreg) { m_aggreg = aggreg; }
    void update(const DSIMem& dsi, Disparity& out, tdv_stream s = nullptr) override {
        tdv_volume v = dsi.abi();
        tdv_image g = dsi.leftOrigin.abi();
        tdv_disparity o = out.abi();
        tdv_volume a;
        if (m_aggreg) a = m_aggreg->abi();
        check(m_ctx.get(), tdv_sgm(m_ctx.get(), &v, dsi.leftOrigin.devMem ? &g : nullptr, &m_params,
                                   m_aggreg ? &a : nullptr, &o, s));
    }

private:
    tdv_sgm_params m_params;
    DSIMem* m_aggreg = nullptr;
};

class SemiGlobalDev : public SemiGlobalOptimizer {
public:
    explicit SemiGlobalDev(Context& ctx) : SemiGlobalOptimizer(ctx, TDV_SEM_REF_GPU) {}
};

class SemiGlobalCPU : public SemiGlobalOptimizer {
public:
    explicit SemiGlobalCPU(Context& ctx) : SemiGlobalOptimizer(ctx, TDV_SEM_REF_CPU) {}
};

class WTADev : public Optimizer {
public:
    explicit WTADev(Context& ctx) : Optimizer(ctx) {}
    void update(const DSIMem& dsi, Disparity& out, tdv_stream s = nullptr) override {
        tdv_volume v = dsi.abi();
        tdv_disparity o = out.abi();
        check(m_ctx.get(), tdv_wta(m_ctx.get(), &v, &o, s));
    }
};

class DynamicProgDev : public Optimizer {
public:
    explicit DynamicProgDev(Context& ctx) : Optimizer(ctx) {}
    void update(const DSIMem& dsi, Disparity& out, tdv_stream s = nullptr) override {
        tdv_volume v = dsi.abi();
        tdv_disparity o = out.abi();
        check(m_ctx.get(), tdv_dp_scanline(m_ctx.get(), &v, &o, s));
    }
};

// ---- matchers without a DSI ----------------------------------------------
// SSD window + WTA (fastwtamatcher.hpp).
class FastWTAMatcher {
public:
    FastWTAMatcher(Context& ctx, int disparityMax, int radius = 3)
        : m_ctx(ctx), m_disparityMax(disparityMax), m_radius(radius) {}
    void update(const FloatImage& left, const FloatImage& right, Disparity& out, tdv_stream s = nullptr) {
        tdv_image l = left.abi(), r = right.abi();
        tdv_disparity o = out.abi();
        check(m_ctx.get(), tdv_fast_wta(m_ctx.get(), &l, &r, m_disparityMax, m_radius, &o, s));
    }

private:
    Context& m_ctx;
    int m_disparityMax, m_radius;
};

// BT cost recomputed inside the aggregation (the role of
// semigloballabmatcher.hpp); u8 inputs with P1/P2 multiples of 1/2 take the
// fused 16-bit path.
class SemiGlobalLabMatcher {
public:
    SemiGlobalLabMatcher(Context& ctx, int disparityMax, float p1 = 10.0f, float p2 = 120.0f, int paths = 8)
        : m_ctx(ctx), m_disparityMax(disparityMax) {
        m_params.p1 = p1;
        m_params.p2 = p2;
        m_params.p2_mode = TDV_P2_CONST;
        m_params.paths = paths;
        m_params.table = TDV_TABLE_FULL;
        m_params.semantics = TDV_SEM_STANDARD;
    }
    void update(const ByteImage& left, const ByteImage& right, Disparity& out, tdv_stream s = nullptr) {
        tdv_image l = left.abi(), r = right.abi();
        tdv_disparity o = out.abi();
        check(m_ctx.get(), tdv_stereo_sgm(m_ctx.get(), &l, &r, m_disparityMax, &m_params, &o, s));
    }

private:
    Context& m_ctx;
    int m_disparityMax;
    tdv_sgm_params m_params;
};

// A cost stage followed by an optimizer stage, as DevStereoMatcher chains
// them (devstereomatcher.cpp:36-48); the DSI is owned by the caller.
class StereoMatcher {
public:
    StereoMatcher(MatchingCost& cost, Optimizer& opt) : m_cost(cost), m_opt(opt) {}
    void update(const FloatImage& left, const FloatImage& right, DSIMem& dsi, Disparity& out,
                tdv_stream s = nullptr) {
        m_cost.update(left, right, dsi, s);
        m_opt.update(dsi, out, s);
    }

private:
    MatchingCost& m_cost;
    Optimizer& m_opt;
};

// ---- stages either side of the matcher -----------------------------------
// A device raster: an 8-bit color frame, a grey image or a disparity map.
// pitchBytes 0 means dense rows.
struct Raster {
    void* devMem = nullptr;
    int width = 0, height = 0, pitchBytes = 0;
    int dtype = TDV_F32;  // TDV_U8, TDV_U16 or TDV_F32
    int channels = 1;     // 1 or 3
    tdv_raster abi() const {
        const int elem = dtype == TDV_U8 ? 1 : dtype == TDV_U16 ? 2 : 4;
        tdv_raster r;
        r.ptr = devMem;
        r.width = width;
        r.height = height;
        r.pitch_bytes = pitchBytes > 0 ? pitchBytes : width * channels * elem;
        r.dtype = dtype;
        r.channels = channels;
        return r;
    }
};

// 8-bit 3-channel frame -> [0,1] grey intensities (width x height floats).
inline void create32FGray(Context& ctx, const Raster& color, float* gray, tdv_stream s = nullptr) {
    tdv_raster c = color.abi();
    check(ctx.get(), tdv_to_gray(ctx.get(), &c, gray, s));
}

// One camera of RectificationCV's calibrated path: the undistort-rectify maps
// are computed once on the device into caller-owned buffers (width x height
// floats each), then every frame is remapped through them.
class Rectifier {
public:
    Rectifier(Context& ctx, float* mapx, float* mapy) : m_ctx(ctx), m_mapx(mapx), m_mapy(mapy) {}
    // K, R, P row-major 3x3 (P's first three columns); dist (k1, k2, p1, p2,
    // k3, k4, k5, k6), zeros for unused terms
    void camera(const double K[9], const double dist[8], const double R[9], const double P[9], int width,
                int height, tdv_stream s = nullptr) {
        check(m_ctx.get(), tdv_rectify_maps(m_ctx.get(), K, dist, R, P, width, height, m_mapx, m_mapy, s));
        m_width = width;
        m_height = height;
    }
    // dst must be width x height (the maps' size), same dtype and channels as src
    void update(const Raster& src, Raster& dst, tdv_stream s = nullptr) const {
        if (dst.width != m_width || dst.height != m_height)
            throw CUException(TDV_ERR_INVALID_ARG, "Rectifier: destination size differs from the maps'");
        tdv_raster a = src.abi(), b = dst.abi();
        check(m_ctx.get(), tdv_remap(m_ctx.get(), &a, m_mapx, m_mapy, &b, s));
    }
    const float* mapx() const { return m_mapx; }
    const float* mapy() const { return m_mapy; }

private:
    Context& m_ctx;
    float *m_mapx, *m_mapy;
    int m_width = -1, m_height = -1;
};

// Pre-filters, FloatImage -> FloatImage (out: width x height floats).
class PreFilter {
public:
    PreFilter(Context& ctx, tdv_filter_kind kind) : m_ctx(ctx), m_kind(kind) {}
    void update(const FloatImage& in, float* out, tdv_stream s = nullptr) {
        tdv_image im = in.abi();
        check(m_ctx.get(), tdv_prefilter(m_ctx.get(), &im, m_kind, out, s));
    }
    // 8-bit input, filtered intensities multiplied by `scale`
    void update(const ByteImage& in, float scale, float* out, tdv_stream s = nullptr) {
        tdv_image im = in.abi();
        im.scale = scale;
        check(m_ctx.get(), tdv_prefilter(m_ctx.get(), &im, m_kind, out, s));
    }

private:
    Context& m_ctx;
    tdv_filter_kind m_kind;
};

class MedianFilterCPU : public PreFilter {
public:
    explicit MedianFilterCPU(Context& ctx) : PreFilter(ctx, TDV_FILTER_GAUSS5) {}
};

class MedianFilterDev : public PreFilter {
public:
    explicit MedianFilterDev(Context& ctx) : PreFilter(ctx, TDV_FILTER_MEDIAN7) {}
};

// Post-filters of a disparity map (F32 or U16, one channel); in and out have
// the same size and dtype and do not overlap.
class PostFilter {
public:
    PostFilter(Context& ctx, tdv_post_kind kind) : m_ctx(ctx), m_kind(kind) {}
    void update(const Raster& in, Raster& out, tdv_stream s = nullptr) {
        tdv_raster a = in.abi(), b = out.abi();
        check(m_ctx.get(), tdv_postfilter(m_ctx.get(), &a, m_kind, &b, s));
    }

private:
    Context& m_ctx;
    tdv_post_kind m_kind;
};

class Dilate : public PostFilter {
public:
    explicit Dilate(Context& ctx) : PostFilter(ctx, TDV_POST_OPEN7) {}
};

// Disparity map -> grid mesh: one vertex (3 floats) per pixel and, when a
// color frame is given, one color (3 floats in [0,1]) per pixel, as
// GLReprojection::updateMesh fills its mesh (device buffers).
class Reprojector {
public:
    virtual ~Reprojector() {}
    void reproject(Context& ctx, const Raster& disp, const Raster* color, float* vertices, float* colors,
                   tdv_stream s = nullptr) const {
        tdv_raster d = disp.abi(), c;
        if (color) c = color->abi();
        tdv_reproject_params p = m_params;
        check(ctx.get(), tdv_reproject(ctx.get(), &d, color ? &c : nullptr, &p, vertices, colors, s));
    }

protected:
    tdv_reproject_params m_params{};
};

class DirectReprojector : public Reprojector {
public:
    explicit DirectReprojector(float zscale = 1.0f) {
        m_params.mode = TDV_REPROJECT_DIRECT;
        m_params.zscale = zscale;
    }
};

class CVReprojector : public Reprojector {
public:
    CVReprojector() { m_params.mode = TDV_REPROJECT_Q; }
    void qmatrix(const float mtx[16]) {
        for (int i = 0; i < 16; i++) m_params.q[i] = mtx[i];
    }
    const float* qmatrix() const { return m_params.q; }
};

// Writes a grid mesh (HOST vertices and optional colors, as Reprojector lays
// them out) to the reference's ASCII PLY.
class PLYMeshExporter {
public:
    explicit PLYMeshExporter(const std::string& name) : m_filename(name) {}
    void exportMesh(const float* vertices, const float* colors, int width, int height) const {
        check(nullptr, tdv_write_ply(m_filename.c_str(), vertices, colors, width, height));
    }
    void filename(const std::string& fname) { m_filename = fname; }
    const std::string& filename() const { return m_filename; }

private:
    std::string m_filename;
};

}  // namespace tdv_b200

#endif  // TDV_STAGES_HPP
