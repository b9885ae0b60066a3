// Drives the C++ stage classes of include/tdv_stages.hpp the way host code
// written against LibThunderVision's stages would.
//
//   stages_demo validate
//       bad arguments must throw CUException before any CUDA call (no GPU
//       needed); exit 0 when every case threw the expected status.
//   stages_demo run W H D left.u8 right.u8 out_prefix
//       BirchfieldCostDev -> SemiGlobalCPU / SemiGlobalDev -> maps, the
//       fused SemiGlobalLabMatcher, FastWTAMatcher and DynamicProgDev on the
//       pair, and the Gaussian-filtered SemiGlobalDev chain; writes
//       out_prefix.{lab,sgm_ref_cpu,sgm_ref_gpu,sgm_filtered,fastwta,dp}.u16
//   stages_demo reconstruct W H D left.rgb right.rgb cams.f64 out_prefix
//       the reference's reconstruction chain from 8-bit 3-channel frames:
//       create32FGray -> Rectifier (both cameras, and the left color frame)
//       -> MedianFilterCPU -> SSDDev + WTADev (d/D map) -> Dilate ->
//       CVReprojector -> PLYMeshExporter.  cams.f64 holds K, dist (8), R, P
//       (3x3) of the left then the right camera, then Q (4x4).  Writes
//       out_prefix.{disp,verts,cols}.f32 and out_prefix.ply
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "tdv_stages.hpp"

using namespace tdv_b200;

static int expect_throw(const char* name, tdv_status want, void (*fn)(Context&), Context& ctx) {
    try {
        fn(ctx);
    } catch (const CUException& e) {
        if (e.status() == want) return 0;
        std::fprintf(stderr, "%s: status %d, want %d (%s)\n", name, (int)e.status(), (int)want, e.what());
        return 1;
    }
    std::fprintf(stderr, "%s: no exception\n", name);
    return 1;
}

static int validate() {
    Context ctx(0);
    int bad = 0;
    bad += expect_throw("null image", TDV_ERR_INVALID_ARG, [](Context& c) {
        BirchfieldCostDev cost(c, 16);
        FloatImage l, r;
        DSIMem dsi;
        cost.update(l, r, dsi);
    }, ctx);
    bad += expect_throw("disparity range", TDV_ERR_UNSUPPORTED, [](Context& c) {
        SemiGlobalLabMatcher m(c, 300);
        static unsigned char fake[64];
        ByteImage l{fake, 8, 8, 8}, r{fake, 8, 8, 8};
        Disparity out;
        static unsigned short d[64];
        out.disp = d;
        m.update(l, r, out);
    }, ctx);
    bad += expect_throw("no outputs", TDV_ERR_INVALID_ARG, [](Context& c) {
        WTADev w(c);
        static float v[64];
        DSIMem dsi;
        dsi.devMem = v;
        dsi.width = 4;
        dsi.height = 4;
        dsi.depth = 4;
        Disparity out;
        w.update(dsi, out);
    }, ctx);
    bad += expect_throw("fast wta radius", TDV_ERR_INVALID_ARG, [](Context& c) {
        FastWTAMatcher f(c, 16, 99);
        static float v[64];
        FloatImage l{v, 8, 8}, r{v, 8, 8};
        static unsigned short d[64];
        Disparity out;
        out.disp = d;
        f.update(l, r, out);
    }, ctx);
    bad += expect_throw("rectifier size", TDV_ERR_INVALID_ARG, [](Context& c) {
        static float mx[64], my[64];
        Rectifier r(c, mx, my);  // no camera yet: any destination size is wrong
        static unsigned char px[64];
        Raster src{px, 8, 8, 0, TDV_U8, 1}, dst{px, 8, 8, 0, TDV_U8, 1};
        r.update(src, dst);
    }, ctx);
    bad += expect_throw("dilate dtype", TDV_ERR_INVALID_ARG, [](Context& c) {
        Dilate d(c);
        static unsigned char a[64], b[64];
        Raster in{a, 8, 8, 0, TDV_U8, 1}, out{b, 8, 8, 0, TDV_U8, 1};
        d.update(in, out);
    }, ctx);
    bad += expect_throw("ply path", TDV_ERR_INVALID_ARG, [](Context&) {
        PLYMeshExporter e("");
        e.exportMesh(nullptr, nullptr, 2, 2);
    }, ctx);
    std::printf(bad ? "validate: FAILED\n" : "validate: ok\n");
    return bad ? 1 : 0;
}

template <typename T>
static T* dev_alloc(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) {
        std::fprintf(stderr, "cudaMalloc failed\n");
        std::exit(2);
    }
    return (T*)p;
}

static std::vector<unsigned char> read_file(const char* path, size_t n) {
    std::vector<unsigned char> b(n);
    FILE* f = std::fopen(path, "rb");
    if (!f || std::fread(b.data(), 1, n, f) != n) {
        std::fprintf(stderr, "cannot read %s\n", path);
        std::exit(2);
    }
    std::fclose(f);
    return b;
}

static void write_map(const std::string& path, const unsigned short* dev, size_t n) {
    std::vector<unsigned short> h(n);
    cudaMemcpy(h.data(), dev, n * 2, cudaMemcpyDeviceToHost);
    FILE* f = std::fopen(path.c_str(), "wb");
    std::fwrite(h.data(), 2, n, f);
    std::fclose(f);
}

static int run(int W, int H, int D, const char* lp, const char* rp, const std::string& out) {
    const size_t n = (size_t)W * H;
    std::vector<unsigned char> lh = read_file(lp, n), rh = read_file(rp, n);
    std::vector<float> lf(n), rf(n);
    const float scale = 1.0f / 255.0f;  // [0,1] intensities by a scale factor (misc.cpp:31)
    for (size_t i = 0; i < n; i++) {
        lf[i] = (float)lh[i] * scale;
        rf[i] = (float)rh[i] * scale;
    }
    unsigned char *l8 = dev_alloc<unsigned char>(n), *r8 = dev_alloc<unsigned char>(n);
    float *l32 = dev_alloc<float>(n), *r32 = dev_alloc<float>(n);
    cudaMemcpy(l8, lh.data(), n, cudaMemcpyHostToDevice);
    cudaMemcpy(r8, rh.data(), n, cudaMemcpyHostToDevice);
    cudaMemcpy(l32, lf.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(r32, rf.data(), n * 4, cudaMemcpyHostToDevice);
    unsigned short* disp = dev_alloc<unsigned short>(n);
    float* vol = dev_alloc<float>(n * D);

    Context ctx(0);
    FloatImage L{l32, W, H}, R{r32, W, H};
    DSIMem dsi;
    dsi.devMem = vol;
    dsi.width = W;
    dsi.height = H;
    dsi.depth = D;
    dsi.layout = TDV_LAYOUT_REF_WHD;
    Disparity o;
    o.disp = disp;

    BirchfieldCostDev bt(ctx, D);
    SemiGlobalCPU sgm_cpu(ctx);
    StereoMatcher m1(bt, sgm_cpu);
    m1.update(L, R, dsi, o);
    write_map(out + ".sgm_ref_cpu.u16", disp, n);

    SemiGlobalDev sgm_gpu(ctx);
    StereoMatcher m2(bt, sgm_gpu);
    m2.update(L, R, dsi, o);
    write_map(out + ".sgm_ref_gpu.u16", disp, n);

    DynamicProgDev dp(ctx);
    dp.update(dsi, o);
    write_map(out + ".dp.u16", disp, n);

    FastWTAMatcher fw(ctx, D, 3);
    fw.update(L, R, o);
    write_map(out + ".fastwta.u16", disp, n);

    SemiGlobalLabMatcher lab(ctx, D, 10.0f, 120.0f, 8);
    ByteImage B8l{l8, W, H, W}, B8r{r8, W, H, W};
    lab.update(B8l, B8r, o);
    write_map(out + ".lab.u16", disp, n);

    // DevStereoMatcher's default chain: Gaussian-filtered pair, SemiGlobalDev
    // with the filtered left image as the P2 guide
    float* filt = dev_alloc<float>(n);
    bt.update(L, R, dsi, filt, TDV_FILTER_GAUSS5);
    sgm_gpu.update(dsi, o);
    write_map(out + ".sgm_filtered.u16", disp, n);
    ctx.deviceStatus();
    std::printf("run: ok\n");
    return 0;
}

template <typename T>
static void write_dev(const std::string& path, const T* dev, size_t n) {
    std::vector<T> h(n);
    cudaMemcpy(h.data(), dev, n * sizeof(T), cudaMemcpyDeviceToHost);
    FILE* f = std::fopen(path.c_str(), "wb");
    std::fwrite(h.data(), sizeof(T), n, f);
    std::fclose(f);
}

static int reconstruct(int W, int H, int D, const char* lp, const char* rp, const char* cp,
                       const std::string& out) {
    const size_t n = (size_t)W * H;
    std::vector<unsigned char> lh = read_file(lp, 3 * n), rh = read_file(rp, 3 * n);
    std::vector<unsigned char> cb = read_file(cp, sizeof(double) * (2 * 35 + 16));
    const double* cams = (const double*)cb.data();
    unsigned char *lc = dev_alloc<unsigned char>(3 * n), *rc = dev_alloc<unsigned char>(3 * n);
    unsigned char* lrect = dev_alloc<unsigned char>(3 * n);
    cudaMemcpy(lc, lh.data(), 3 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(rc, rh.data(), 3 * n, cudaMemcpyHostToDevice);
    float *gray = dev_alloc<float>(n), *grect[2] = {dev_alloc<float>(n), dev_alloc<float>(n)};
    float *filt[2] = {dev_alloc<float>(n), dev_alloc<float>(n)};
    float *maps[4] = {dev_alloc<float>(n), dev_alloc<float>(n), dev_alloc<float>(n), dev_alloc<float>(n)};
    float *vol = dev_alloc<float>(n * D), *disp = dev_alloc<float>(n), *opened = dev_alloc<float>(n);
    float *verts = dev_alloc<float>(3 * n), *cols = dev_alloc<float>(3 * n);

    Context ctx(0);
    Rectifier rect[2] = {Rectifier(ctx, maps[0], maps[1]), Rectifier(ctx, maps[2], maps[3])};
    unsigned char* frames[2] = {lc, rc};
    for (int c = 0; c < 2; c++) {
        const double* k = cams + 35 * c;
        rect[c].camera(k, k + 9, k + 17, k + 26, W, H);
        Raster color{frames[c], W, H, 0, TDV_U8, 3};
        create32FGray(ctx, color, gray);
        Raster g{gray, W, H, 0, TDV_F32, 1}, gr{grect[c], W, H, 0, TDV_F32, 1};
        rect[c].update(g, gr);
        MedianFilterCPU gauss(ctx);
        gauss.update(FloatImage{grect[c], W, H}, filt[c]);
    }
    Raster lcol{lc, W, H, 0, TDV_U8, 3}, lrc{lrect, W, H, 0, TDV_U8, 3};
    rect[0].update(lcol, lrc);

    SSDDev ssd(ctx, D);
    WTADev wta(ctx);
    StereoMatcher matcher(ssd, wta);
    DSIMem dsi;
    dsi.devMem = vol;
    dsi.width = W;
    dsi.height = H;
    dsi.depth = D;
    dsi.layout = TDV_LAYOUT_HWD;
    Disparity o;
    o.dispNorm = disp;
    matcher.update(FloatImage{filt[0], W, H}, FloatImage{filt[1], W, H}, dsi, o);

    Dilate dilate(ctx);
    Raster din{disp, W, H, 0, TDV_F32, 1}, dout{opened, W, H, 0, TDV_F32, 1};
    dilate.update(din, dout);

    CVReprojector repr;
    float q[16];
    for (int i = 0; i < 16; i++) q[i] = (float)cams[70 + i];
    repr.qmatrix(q);
    repr.reproject(ctx, dout, &lrc, verts, cols);
    ctx.deviceStatus();

    write_dev(out + ".disp.f32", opened, n);
    write_dev(out + ".verts.f32", verts, 3 * n);
    write_dev(out + ".cols.f32", cols, 3 * n);
    std::vector<float> hv(3 * n), hc(3 * n);
    cudaMemcpy(hv.data(), verts, 3 * n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hc.data(), cols, 3 * n * 4, cudaMemcpyDeviceToHost);
    PLYMeshExporter(out + ".ply").exportMesh(hv.data(), hc.data(), W, H);
    std::printf("reconstruct: ok\n");
    return 0;
}

int main(int argc, char** argv) {
    if (argc >= 2 && std::strcmp(argv[1], "validate") == 0) return validate();
    if (argc == 8 && std::strcmp(argv[1], "run") == 0)
        return run(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]), argv[5], argv[6], argv[7]);
    if (argc == 9 && std::strcmp(argv[1], "reconstruct") == 0)
        return reconstruct(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]), argv[5], argv[6], argv[7],
                           argv[8]);
    std::fprintf(stderr,
                 "usage: stages_demo validate | run W H D left.u8 right.u8 out_prefix |"
                 " reconstruct W H D left.rgb right.rgb cams.f64 out_prefix\n");
    return 2;
}
