// Harness around the reference's own CPU aggregation code -- TEST
// INFRASTRUCTURE ONLY.  oracle/Makefile's `ref` target compiles, where they
// lie in the reference tree, LibThunderVision's semiglobalcpu.cpp
// (costPath, SemiGlobalCPU::updateImpl), wtacpu.cpp (WTACPU::wta) and
// semiglobal.cu (the SGPaths table builders), with the stand-in headers of
// oracle/ref_shim/, and links them with this file into oracle/_ref/libtdvref.so.
// The oracle's tests compare the oracle (tdv_oracle.cpp) with it bit for bit.
//
// This file supplies what the reference's image and volume classes keep in
// other translation units (dsimem.cpp, floatimage.cpp, optimizer.cpp,
// benchmark.cpp), over host arrays, and a C entry point per function.  The
// member definitions follow the declarations in the reference headers: a
// DSIMem holds a W x H x D float volume in the reference layout
// ((x*H)+y)*D+d and toCpuMem() returns a new[]-allocated copy of it
// (tdvision/dsimem.cpp:55-83 copies the device volume the same way); a
// FloatImage holds a W x H float image whose CvMat data the optimizer reads
// as its intensity image and overwrites with d/D (tdvision/semiglobalcpu.cpp:200,
// wtacpu.cpp:35-36).
#include <cstdint>
#include <cstring>
#include <vector>

#include "cudaconstraits.hpp"
#include "cuerr.hpp"
#include "semiglobal.h"
#include "semiglobalcpu.hpp"
#include "wtacpu.hpp"

namespace tdv {

// ---- volume and image classes over host memory
LocalDSIMem::LocalDSIMem(size_t typeSize) : m_dim(0), m_typeSize(typeSize) {
    m_mem.ptr = nullptr;
    m_mem.pitch = 0;
    m_mem.xsize = m_mem.ysize = 0;
}
LocalDSIMem::~LocalDSIMem() { unalloc(); }
cudaPitchedPtr LocalDSIMem::mem(const Dim& dim) {
    if (dim != m_dim) {
        unalloc();
        m_dim = dim;
        m_mem.ptr = new unsigned char[dim.size() * m_typeSize]();
        m_mem.pitch = dim.depth() * m_typeSize;
        m_mem.xsize = dim.depth();
        m_mem.ysize = dim.height();
    }
    return m_mem;
}
void LocalDSIMem::unalloc() {
    delete[] (unsigned char*)m_mem.ptr;
    m_mem.ptr = nullptr;
    m_dim = Dim(0);
}
void* LocalDSIMem::toCpuMem() {
    unsigned char* cpu = new unsigned char[m_dim.size() * m_typeSize];
    std::memcpy(cpu, m_mem.ptr, m_dim.size() * m_typeSize);
    return cpu;
}
void DSIMemImpl::init(const Dim& dim, FloatImage lorigin) {
    m_dsiMem.mem(dim);
    m_leftOrigin = lorigin;
}
DSIMem DSIMem::Create(const Dim& dim, FloatImage lorigin) {
    DSIMemImpl* impl = new DSIMemImpl;
    impl->init(dim, lorigin);
    return DSIMem(impl);
}

FloatImageImpl::FloatImageImpl() : m_cpuMem(nullptr), m_syncDev(-1), m_dim(0) {}
void FloatImageImpl::initCPU(const Dim& dim) {
    m_dim = dim;
    m_cpuMem = new CvMat();
    m_cpuMem->rows = (int)dim.height();
    m_cpuMem->cols = (int)dim.width();
    m_cpuMem->step = (int)(dim.width() * sizeof(float));
    m_cpuMem->data.fl = new float[dim.size()]();
}
CvMat* FloatImageImpl::cpuMem() { return m_cpuMem; }
void FloatImageImpl::dispose() {
    if (m_cpuMem) {
        delete[] m_cpuMem->data.fl;
        delete m_cpuMem;
        m_cpuMem = nullptr;
    }
}

// ---- pipeline base and timing: nothing to do on the host here
AbstractOptimizer::AbstractOptimizer() : m_rpipe(nullptr) {}
bool AbstractOptimizer::update() { return false; }
void CudaBenchmarker::begin() {}
void CudaBenchmarker::end() {}

// Named by the device launcher SemiGlobalDevRun in semiglobal.cu, which the
// oracle never calls (no GPU work happens here).
void CUerrExpPol::report(const char*) {}
WorkSize CudaConstraits::imageWorkSize(const Dim&) { return WorkSize(dim3(1), dim3(1)); }
void WTARunDev(const Dim&, cudaPitchedPtr, float*) {}

// defined in semiglobalcpu.cpp (no header declares it)
void costPath(const Dim& dsiDim, const float* dsi, const float* img, const SGPoint& start, const sSGPoint& dir,
              size_t pathLength, float* aggregVol, float* lastCost, float* newCost);

}  // namespace tdv

namespace {

// SemiGlobalCPU with its protected update callable.
struct RunSemiGlobalCPU : tdv::SemiGlobalCPU {
    void run(tdv::DSIMem m, tdv::FloatImage i) { updateImpl(m, i); }
};

}  // namespace

extern "C" {

// SGPaths::getDescCPU (tdvision/semiglobal.cu:57-81): rows of (sx, sy, ex, ey,
// dx, dy, size); returns the path count.
int ref_path_table(int W, int H, int32_t* out) {
    size_t n = 0;
    tdv::SGPath* p = tdv::SGPaths::getDescCPU(tdv::Dim(W, H), &n);
    if (out)
        for (size_t i = 0; i < n; i++) {
            int32_t* r = out + 7 * i;
            r[0] = p[i].start.x;
            r[1] = p[i].start.y;
            r[2] = p[i].end.x;
            r[3] = p[i].end.y;
            r[4] = p[i].dir.x;
            r[5] = p[i].dir.y;
            r[6] = p[i].size;
        }
    delete[] p;
    return (int)n;
}

// SemiGlobalCPU::updateImpl (tdvision/semiglobalcpu.cpp:173-230) on a cost
// DSI in the reference layout, with `img` (W x H) as the optimizer's image:
// writes the disparity map d/D it leaves in that image.
void ref_semiglobal_cpu(const float* dsi, int W, int H, int D, const float* img, float* disp_norm) {
    tdv::FloatImage im = tdv::FloatImage::CreateCPU(tdv::Dim(W, H));
    std::memcpy(im.cpuMem()->data.fl, img, sizeof(float) * (size_t)W * H);
    tdv::DSIMem mem = tdv::DSIMem::Create(tdv::Dim(W, H, D), im);
    std::memcpy(mem.mem().ptr, dsi, sizeof(float) * (size_t)W * H * D);
    RunSemiGlobalCPU opt;
    opt.run(mem, im);  // updateImpl keeps (and never frees) its toCpuMem copy, as in the reference
    std::memcpy(disp_norm, im.cpuMem()->data.fl, sizeof(float) * (size_t)W * H);
}

// The aggregated volume of updateImpl's loop: the reference's costPath over
// its table, forward from each path's start, then backward from its end,
// into a zeroed volume (tdvision/semiglobalcpu.cpp:183-222).
void ref_semiglobal_cpu_volume(const float* dsi, int W, int H, int D, const float* img, float* aggreg) {
    const tdv::Dim dim(W, H, D);
    size_t n = 0;
    tdv::SGPath* paths = tdv::SGPaths::getDescCPU(tdv::Dim(W, H), &n);
    std::memset(aggreg, 0, sizeof(float) * dim.size());
    std::vector<float> last(D + 2), next(D + 2);
    last[0] = next[0] = last[D + 1] = next[D + 1] = std::numeric_limits<float>::infinity();
    for (size_t p = 0; p < n; p++) {
        tdv::costPath(dim, dsi, img, paths[p].start, paths[p].dir, paths[p].size, aggreg, last.data(), next.data());
        const tdv::sSGPoint inv = {(short)-paths[p].dir.x, (short)-paths[p].dir.y};
        tdv::costPath(dim, dsi, img, paths[p].end, inv, paths[p].size, aggreg, last.data(), next.data());
    }
    delete[] paths;
}

// WTACPU::wta (tdvision/wtacpu.cpp:14-39) on a volume in the reference layout.
void ref_wta(const float* dsi, int W, int H, int D, float* disp_norm) {
    tdv::WTACPU::wta(tdv::Dim(W, H, D), dsi, disp_norm);
}

}  // extern "C"
