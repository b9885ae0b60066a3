// CPU ORACLE for the dense-stereo hot path -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of LibThunderVision's matching-cost / aggregation /
// reduction algorithms.  Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg load this library, and only as the checker (or as the timed
// CPU arm).  The product path (thundervision_b200) never links or calls it.
//
// Each function cites the reference lines it restates (paths relative to the
// ThunderVision project root; tdvision/ = LibThunderVision/src/tdvision/).
// The reference publishes no golden vectors for this path: parity of this
// oracle is pinned by hand-computed known-answer tests (tests/golden) and by
// reading the reference sources line by line.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off -fopenmp).  Contraction is
// off so that every float expression rounds exactly as written.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const float kInf = std::numeric_limits<float>::infinity();

enum { LAYOUT_REF_WHD = 0, LAYOUT_HWD = 1 };
enum { SEM_STANDARD = 0, SEM_REF_CPU = 1, SEM_REF_GPU = 2 };
enum { TABLE_FULL = 0, TABLE_REF = 1 };
enum { P2_CONST = 0, P2_ADJUST = 1 };

struct Geo {
    int W, H, D, layout;
    // Offset of cell (x, y, d).  REF_WHD is the reference DSI layout
    // ((x*H)+y)*D+d (tdvision/semiglobalcpu.cpp:18-22, dsimemutil.h:6);
    // HWD is row-major ((y*W)+x)*D+d.
    inline size_t off(int x, int y, int d) const {
        if (layout == LAYOUT_REF_WHD)
            return ((size_t)x * H + y) * (size_t)D + d;
        return ((size_t)y * W + x) * (size_t)D + d;
    }
};

// Point-sampled texture fetch with unnormalised coordinates.  The reference
// binds cudaAddressModeWrap with normalized = false
// (tdvision/birchfieldcost.cu:160-163); wrap is defined only for normalised
// coordinates, so out-of-range taps read the edge texel (clamp).
inline float tex(const float* img, int W, int H, int x, int y) {
    x = x < 0 ? 0 : (x >= W ? W - 1 : x);
    y = y < 0 ? 0 : (y >= H ? H - 1 : y);
    return img[(size_t)y * W + x];
}

// CUDA's float min/max (fminf/fmaxf).
inline float fmn(float a, float b) { return std::fmin(a, b); }
inline float fmx(float a, float b) { return std::fmax(a, b); }
// std::min / std::max: (b < a) ? b : a.
inline float smin(float a, float b) { return (b < a) ? b : a; }

// An image with its own size: taps clamp to each image's own edges (the DSI
// takes the smaller size, tdvision/matchingcost.cpp:20-24).
struct Img {
    const float* p;
    int W, H;
    float at(int x, int y) const { return tex(p, W, H, x, y); }
};

// tdvision/birchfieldcost.cu:14-39 (costAtDisp), one tap (v == x).
float bt_at(const Img& L, const Img& R, int x, int y, int disp) {
    float sum = 0.0f;
    const float lI = L.at(x, y);
    const float rI = R.at(x - disp, y);
    const float laI = 0.5f * (lI + L.at(x - 1, y));
    const float lbI = 0.5f * (lI + L.at(x + 1, y));
    const float raI = 0.5f * (rI + R.at(x - disp - 1, y));
    const float rbI = 0.5f * (rI + R.at(x - disp + 1, y));
    const float lImi = fmn(laI, fmn(lbI, lI));
    const float lIma = fmx(laI, fmx(lbI, lI));
    const float rImi = fmn(raI, fmn(rbI, rI));
    const float rIma = fmx(raI, fmx(rbI, rI));
    sum += fmn(fmx(0.0f, fmx(lI - rIma, rImi - lI)),
               fmx(0.0f, fmx(rI - lIma, lImi - rI)));
    return sum;
}

// tdvision/ssd.cu:15-29 (ssdAtDisp): rows then columns in [-r, r].
float ssd_at(const Img& L, const Img& R, int x, int y, int disp, int r) {
    float sum = 0.0f;
    for (int row = -r; row <= r; row++)
        for (int col = -r; col <= r; col++) {
            const float lI = L.at(x + col, y + row);
            const float rI = R.at(x + col - disp, y + row);
            const float df = lI - rI;
            const float sq = df * df;
            sum = sum + sq;
        }
    return sum;
}

// tdvision/crosscorrelation.cu:11-28 (ccAtDisp): un-centred NCC.
float ncc_at(const Img& L, const Img& R, int x, int y, int disp, int r) {
    float dom = 0.0f, ls = 0.0f, rs = 0.0f;
    for (int row = -r; row <= r; row++)
        for (int col = -r; col <= r; col++) {
            const float lv = L.at(x + col, y + row);
            const float rv = R.at(x + col - disp, y + row);
            const float lr = lv * rv;
            const float ll = lv * lv;
            const float rr = rv * rv;
            dom = dom + lr;
            ls = ls + ll;
            rs = rs + rr;
        }
    const float prod = ls * rs;
    const float den = std::sqrt(prod);
    const float q = dom / den;
    return 1.0f - q;
}

struct Walk {
    int sx, sy, ex, ey, dx, dy, size;
};

// tdvision/semiglobal.cu:57-81 (getDescCPU) and the four descriptor builders
// :116-230.  TABLE_REF reproduces the entries exactly as written, including the
// stale `end` of the diagonal entries that overshoot the short image side
// (:163-166, :197-205).  TABLE_FULL recomputes every end as
// start + (size-1)*dir.
std::vector<Walk> path_table(int W, int H, int table) {
    const int lastX = W - 1, lastY = H - 1;
    std::vector<Walk> p;
    p.reserve((size_t)W + H + 2 * ((size_t)W + H - 1));
    // horizontalPathsDesc :116-130
    for (int i = 0; i < H; i++) p.push_back({0, i, W - 1, i, 1, 0, W});
    // verticalPathsDesc :132-146
    for (int i = 0; i < W; i++) p.push_back({i, 0, i, H - 1, 0, 1, H});
    // bottomTopDiagonalDesc :154-185, direction (1,1)
    for (int i = 0; i < W; i++) {
        Walk w;
        w.sx = lastX - i; w.sy = 0;
        w.ex = lastX; w.ey = std::min(i, lastY);
        w.size = w.ey - w.sy + 1;
        w.dx = 1; w.dy = 1;
        p.push_back(w);
    }
    for (int i = 0; i < H - 1; i++) {
        Walk w;
        w.sx = 0; w.sy = i + 1;
        w.ex = std::min(lastY - (i + 1), lastX); w.ey = lastY;
        w.size = w.ex - w.sx + 1;
        w.dx = 1; w.dy = 1;
        p.push_back(w);
    }
    // topBottomDiagonaDesc :191-230, direction (-1,1)
    for (int i = 0; i < W; i++) {
        const int diag = std::min(i + 1, H);
        p.push_back({i, 0, 0, diag - 1, -1, 1, diag});
    }
    for (int i = 0; i < H - 1; i++) {
        const int sX = lastX, sY = i + 1;
        const int diag = std::min(H - (i + 1), W);
        p.push_back({sX, sY, sX - diag + 1, sY + diag - 1, -1, 1, diag});
    }
    if (table == TABLE_FULL)
        for (auto& w : p) {
            w.ex = w.sx + (w.size - 1) * w.dx;
            w.ey = w.sy + (w.size - 1) * w.dy;
        }
    return p;
}

struct SgmCfg {
    float p1, p2;
    int p2_mode, sem;
};

// One path walk: tdvision/semiglobalcpu.cpp:56-126 (costPath, REF_CPU), with
// the deltas of the device kernel tdvision/semiglobal.cu:283-466 (REF_GPU)
// and the plain SGM recurrence (STANDARD).
//   REF_CPU : start cell assigns S = C (:81); previous = C (:82); the minimum
//             over d scans lastCost[0..D-1] = {sentinel, L(0..D-2)} with the
//             CUDA host min(float,float) = fminf (:95-97); min4 is the
//             std::min chain (:39, :115-119).
//   REF_GPU : start accumulates (semiglobal.cu:355,361); previous = C + P1
//             while the running minimum starts from C (:353-354); fminf
//             everywhere (:320); full minimum over d.
//   STANDARD: start accumulates; previous = C; fminf; full minimum over d.
// P2 is constant or P2/|I(p)-I(p-r)| (semiglobalcpu.cpp:99-102).
void cost_path(const Geo& g, const float* C, const float* img, const SgmCfg& cfg,
               int sx, int sy, int dx, int dy, int len, float* S,
               std::vector<float>& last, std::vector<float>& nxt, std::vector<float>& lastMin) {
    const int D = g.D;
    int X = sx, Y = sy;
    last[0] = kInf; last[D + 1] = kInf;
    nxt[0] = kInf; nxt[D + 1] = kInf;
    float lastI = img[(size_t)Y * g.W + X];
    for (int z = 0; z < D; z++) {
        const size_t o = g.off(X, Y, z);
        const float c = C[o];
        if (cfg.sem == SEM_REF_CPU) S[o] = c; else S[o] = S[o] + c;
        last[z + 1] = (cfg.sem == SEM_REF_GPU) ? c + cfg.p1 : c;
        lastMin[z] = c;
    }
    for (int step = 1; step < len; step++) {
        X += dx; Y += dy;
        float m;
        if (cfg.sem == SEM_REF_CPU) {
            m = last[0];
            for (int z = 1; z < D; z++) m = fmn(last[z], m);
        } else if (cfg.sem == SEM_REF_GPU) {
            m = kInf;
            for (int z = 0; z < D; z++) m = fmn(m, lastMin[z]);
        } else {
            m = kInf;
            for (int z = 0; z < D; z++) m = fmn(m, last[z + 1]);
        }
        const float I = img[(size_t)Y * g.W + X];
        float p2a = cfg.p2;
        if (cfg.p2_mode == P2_ADJUST) {
            const float df = std::fabs(I - lastI);
            p2a = cfg.p2 / df;
        }
        lastI = I;
        const float mp2 = m + p2a;
        for (int z = 0; z < D; z++) {
            const size_t o = g.off(X, Y, z);
            const float c = C[o];
            const float a = last[z + 1];
            const float b = last[z] + cfg.p1;
            const float e = last[z + 2] + cfg.p1;
            float mn;
            if (cfg.sem == SEM_REF_CPU) mn = smin(a, smin(b, smin(e, mp2)));
            else mn = fmn(a, fmn(b, fmn(e, mp2)));
            const float t = c + mn;
            const float Lr = t - m;
            S[o] = S[o] + Lr;
            nxt[z + 1] = Lr;
            lastMin[z] = Lr;
        }
        std::swap(last, nxt);
    }
}

bool family_enabled(int dx, int dy, int paths) {
    if (paths == 8) return true;
    return dx == 0 || dy == 0;  // 4-path: horizontal and vertical only
}

}  // namespace

extern "C" {

int orc_version() { return 4; }

// Grey u8 -> float intensity: v * scale (scale = 1 for the integer domain,
// 1/255 for the reference domain of misc.cpp:31-32).
void orc_u8_to_f32(const uint8_t* src, size_t n, float scale, float* dst) {
    for (size_t i = 0; i < n; i++) dst[i] = (float)src[i] * scale;
}

// tdvision/birchfieldcost.cu:41-59 (birchfieldKernTexture): INF where x-d<0.
void orc_bt_cost(const float* L, const float* R, int W, int H, int D, int layout, float* out) {
    Geo g{W, H, D, layout};
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int d = 0; d < D; d++)
                out[g.off(x, y, d)] = (x - d >= 0) ? bt_at(Img{L, W, H}, Img{R, W, H}, x, y, d) : kInf;
}

// tdvision/ssd.cu:32-50 (ssdKern): INF where x-d<0; window radius r (3 = 7x7).
void orc_ssd_cost(const float* L, const float* R, int W, int H, int D, int r, int layout, float* out) {
    Geo g{W, H, D, layout};
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int d = 0; d < D; d++)
                out[g.off(x, y, d)] = (x - d >= 0) ? ssd_at(Img{L, W, H}, Img{R, W, H}, x, y, d, r) : kInf;
}

// tdvision/crosscorrelation.cu:30-49 (ccorrelationKern): nDisps = min(D, x+1),
// INF beyond; window radius r (1 = 3x3).
void orc_ncc_cost(const float* L, const float* R, int W, int H, int D, int r, int layout, float* out) {
    Geo g{W, H, D, layout};
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int d = 0; d < D; d++)
                out[g.off(x, y, d)] = (d < x + 1) ? ncc_at(Img{L, W, H}, Img{R, W, H}, x, y, d, r) : kInf;
}

// Any of the three costs for a pair of different sizes: the DSI is the
// smaller width x height, each image's taps clamp to its own edges.
// kind: 0 BT, 1 SSD, 2 NCC (tdv_cost_kind).
void orc_cost_pair(const float* L, int LW, int LH, const float* R, int RW, int RH, int D, int kind, int r,
                   int layout, float* out) {
    const int W = std::min(LW, RW), H = std::min(LH, RH);
    Geo g{W, H, D, layout};
    const Img li{L, LW, LH}, ri{R, RW, RH};
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int d = 0; d < D; d++) {
                float v = kInf;
                if (x - d >= 0)
                    v = kind == 0 ? bt_at(li, ri, x, y, d) : kind == 1 ? ssd_at(li, ri, x, y, d, r)
                                                                       : ncc_at(li, ri, x, y, d, r);
                out[g.off(x, y, d)] = v;
            }
}

int orc_path_count(int W, int H) { return W + H + 2 * (W + H - 1); }

// Path table as int32 rows {sx, sy, ex, ey, dx, dy, size}.
void orc_path_table(int W, int H, int table, int32_t* out) {
    auto p = path_table(W, H, table);
    for (size_t i = 0; i < p.size(); i++) {
        const Walk& w = p[i];
        int32_t* o = out + 7 * i;
        o[0] = w.sx; o[1] = w.sy; o[2] = w.ex; o[3] = w.ey;
        o[4] = w.dx; o[5] = w.dy; o[6] = w.size;
    }
}

// tdvision/wtacpu.cpp:14-39: strict '<' from d = 0, so ties go to the lowest d;
// output float(d)/float(D).
void orc_wta(const float* V, int layout, int W, int H, int D, float* disp_norm, uint16_t* disp) {
    Geo g{W, H, D, layout};
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            float best = kInf;
            int bd = 0;
            for (int d = 0; d < D; d++) {
                const float v = V[g.off(x, y, d)];
                if (v < best) { best = v; bd = d; }
            }
            if (disp_norm) disp_norm[(size_t)W * y + x] = float(bd) / float(D);
            if (disp) disp[(size_t)W * y + x] = (uint16_t)bd;
        }
}

// Aggregation: tdvision/semiglobalcpu.cpp:173-230 (SemiGlobalCPU::updateImpl).
// Walks the path table in order, forward from `start` then backward from `end`
// along -dir (:210-222), then WTA (:225).  The aggregation volume starts at
// zero (the reference's zeroVolume at :41-54 swaps x and y and relies on fresh
// zero pages; zero-initialising is its effect).  `guide` is the intensity image
// for P2 adjustment; the reference reads the freshly created output image there
// (:200 with optimizer.cpp:18-19) and the left image is substituted.
// threads > 1 runs the walks of one direction concurrently.  That preserves
// the per-cell order of the sequential loop for the FULL table and for
// landscape/square REF tables (whose repeated reverse walks follow their own
// forward walk); portrait REF tables always run sequentially.
void orc_sgm(const float* C, int layout, const float* guide, int W, int H, int D,
             float p1, float p2, int p2_mode, int paths, int table, int sem, int threads,
             float* S_out, float* disp_norm, uint16_t* disp) {
    Geo g{W, H, D, layout};
    const size_t n = (size_t)W * H * D;
    std::vector<float> Sv;
    float* S = S_out;
    if (!S) { Sv.assign(n, 0.0f); S = Sv.data(); }
    else std::memset(S, 0, n * sizeof(float));
    SgmCfg cfg{p1, p2, p2_mode, sem};
    auto tab = path_table(W, H, table);
    const bool parallel = threads > 1 && !(table == TABLE_REF && H > W);
    if (!parallel) {
        std::vector<float> a(D + 2), b(D + 2), m(D);
        for (const Walk& w : tab) {
            if (!family_enabled(w.dx, w.dy, paths)) continue;
            cost_path(g, C, guide, cfg, w.sx, w.sy, w.dx, w.dy, w.size, S, a, b, m);
            cost_path(g, C, guide, cfg, w.ex, w.ey, -w.dx, -w.dy, w.size, S, a, b, m);
        }
    } else {
        // families are contiguous in the table: H [0,H), V [H,H+W), D1, D2
        const size_t fam[5] = {0, (size_t)H, (size_t)H + W, (size_t)H + W + (W + H - 1),
                               tab.size()};
#ifdef _OPENMP
        omp_set_num_threads(threads);
#endif
        for (int f = 0; f < 4; f++) {
            if (!family_enabled(tab[fam[f]].dx, tab[fam[f]].dy, paths)) continue;
            for (int rev = 0; rev < 2; rev++) {
#pragma omp parallel
                {
                    std::vector<float> a(D + 2), b(D + 2), m(D);
                    // Repeated identical reverse walks (stale REF ends) touch
                    // the same cells; they are handled by the one thread that
                    // owns the first of them, in table order.
#pragma omp for schedule(dynamic, 8)
                    for (long i = (long)fam[f]; i < (long)fam[f + 1]; i++) {
                        const Walk& w = tab[i];
                        if (rev == 0) {
                            cost_path(g, C, guide, cfg, w.sx, w.sy, w.dx, w.dy, w.size, S, a, b, m);
                            continue;
                        }
                        bool first = true;
                        for (long j = (long)fam[f]; j < i; j++) {
                            const Walk& v = tab[j];
                            if (v.ex == w.ex && v.ey == w.ey && v.size == w.size) { first = false; break; }
                        }
                        if (!first) continue;
                        for (long j = i; j < (long)fam[f + 1]; j++) {
                            const Walk& v = tab[j];
                            if (j == i || (v.ex == w.ex && v.ey == w.ey && v.size == w.size))
                                cost_path(g, C, guide, cfg, v.ex, v.ey, -v.dx, -v.dy, v.size, S, a, b, m);
                        }
                    }
                }
            }
        }
    }
    orc_wta(S, layout, W, H, D, disp_norm, disp);
}

// Left-right consistency (no reference counterpart).  Right disparity
// dR(xr) = argmin_d S(xr+d, y, d) over xr+d < W (lowest d on ties); a left
// pixel is invalid (0xFFFF) when x-dL < 0 or |dL - dR(x-dL)| > thr.
void orc_lr_check(const float* S, int layout, int W, int H, int D, int thr,
                  uint16_t* dispL, uint16_t* dispR) {
    Geo g{W, H, D, layout};
    std::vector<uint16_t> dr((size_t)W);
    for (int y = 0; y < H; y++) {
        for (int xr = 0; xr < W; xr++) {
            float best = kInf;
            int bd = 0;
            for (int d = 0; d < D && xr + d < W; d++) {
                const float v = S[g.off(xr + d, y, d)];
                if (v < best) { best = v; bd = d; }
            }
            dr[xr] = (uint16_t)bd;
            if (dispR) dispR[(size_t)W * y + xr] = (uint16_t)bd;
        }
        for (int x = 0; x < W; x++) {
            uint16_t& dl = dispL[(size_t)W * y + x];
            const int xr = x - (int)dl;
            if (xr < 0 || std::abs((int)dl - (int)dr[xr]) > thr) dl = 0xFFFF;
        }
    }
}

// Dynamic-programming scanline: the recurrence of
// tdvision/dynamicprogcpu.cpp:13-62 (A = C + min over d-1/d/d+1 with the tie
// codes -1/0/+1 of :48-57, no penalty) and the backtrack of
// tdvision/dynamicprog.cu:68-101 with its row indexing fixed: argmin of the
// row's last column (lowest d), then from x = W-1 down to 0 follow the code
// stored at (x, d) and write the reached d at x.
void orc_dp(const float* C, int layout, int W, int H, int D, float* disp_norm, uint16_t* disp) {
    Geo g{W, H, D, layout};
#pragma omp parallel
    {
        std::vector<float> A((size_t)W * D);
        std::vector<int8_t> P((size_t)W * D);
#pragma omp for schedule(static)
        for (int y = 0; y < H; y++) {
            for (int z = 0; z < D; z++) { A[z] = C[g.off(0, y, z)]; P[z] = 0; }
            for (int x = 1; x < W; x++) {
                const float* Ap = &A[(size_t)(x - 1) * D];
                for (int z = 0; z < D; z++) {
                    const float c0 = C[g.off(x, y, z)];
                    const float c1 = z > 0 ? Ap[z - 1] : kInf;
                    const float c2 = Ap[z];
                    const float c3 = z < D - 1 ? Ap[z + 1] : kInf;
                    float m; int8_t p;
                    if (c1 < c2 && c1 < c3) { m = c1; p = -1; }
                    else if (c2 < c3) { m = c2; p = 0; }
                    else { m = c3; p = 1; }
                    A[(size_t)x * D + z] = c0 + m;
                    P[(size_t)x * D + z] = p;
                }
            }
            const float* Al = &A[(size_t)(W - 1) * D];
            int z = 0;
            float mn = Al[0];
            for (int k = 1; k < D; k++) if (Al[k] < mn) { mn = Al[k]; z = k; }
            for (int x = W - 1; x >= 0; x--) {
                const int nz = z + P[(size_t)x * D + z];
                if (nz >= 0 && nz < D) z = nz;
                if (disp_norm) disp_norm[(size_t)W * y + x] = float(z) / float(D);
                if (disp) disp[(size_t)W * y + x] = (uint16_t)z;
            }
        }
    }
}

// tdvision/fastwta.cu:32-53 (fastWtaKern): SSD window radius r, candidates
// d < min(D, x+1), strict '<' (lowest d).
void orc_fastwta(const float* L, const float* R, int W, int H, int D, int r,
                 float* disp_norm, uint16_t* disp) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            float best = kInf;
            int bd = 0;
            const int nd = std::min(D, x + 1);
            for (int d = 0; d < nd; d++) {
                const float v = ssd_at(Img{L, W, H}, Img{R, W, H}, x, y, d, r);
                if (v < best) { best = v; bd = d; }
            }
            if (disp_norm) disp_norm[(size_t)W * y + x] = float(bd) / float(D);
            if (disp) disp[(size_t)W * y + x] = (uint16_t)bd;
        }
}

// ---------------------------------------------------------------------------
// Soft-argmin SGM in FP64 (no reference counterpart): the STANDARD recurrence
// over the FULL table with constant P2, S = sum over directions,
// p_d = softmax(-S/tau), dhat = sum_d d*p_d.  Cost volume layout HWD.
// The adjoint routes each path gradient through the chosen min-plus argument
// (ties: same d, then d-1, then d+1, then the P2 jump) and through the -m
// term to the lowest argmin of the previous step.

namespace {

struct DWalk { int sx, sy, dx, dy, len; };

std::vector<DWalk> soft_walks(int W, int H, int paths) {
    std::vector<DWalk> ws;
    auto tab = path_table(W, H, TABLE_FULL);
    for (const Walk& w : tab) {
        if (!family_enabled(w.dx, w.dy, paths)) continue;
        ws.push_back({w.sx, w.sy, w.dx, w.dy, w.size});
        ws.push_back({w.ex, w.ey, -w.dx, -w.dy, w.size});
    }
    return ws;
}

void soft_path_forward(const double* C, int W, int D, double p1, double p2, const DWalk& w,
                       std::vector<double>& Lbuf) {
    const double inf = std::numeric_limits<double>::infinity();
    Lbuf.assign((size_t)w.len * D, 0.0);
    int X = w.sx, Y = w.sy;
    for (int z = 0; z < D; z++) Lbuf[z] = C[((size_t)Y * W + X) * D + z];
    for (int t = 1; t < w.len; t++) {
        X += w.dx; Y += w.dy;
        const double* Lp = &Lbuf[(size_t)(t - 1) * D];
        double m = inf;
        for (int z = 0; z < D; z++) m = std::fmin(m, Lp[z]);
        for (int z = 0; z < D; z++) {
            const double a = Lp[z];
            const double b = z > 0 ? Lp[z - 1] + p1 : inf;
            const double e = z < D - 1 ? Lp[z + 1] + p1 : inf;
            const double mn = std::fmin(a, std::fmin(b, std::fmin(e, m + p2)));
            Lbuf[(size_t)t * D + z] = C[((size_t)Y * W + X) * D + z] + mn - m;
        }
    }
}

}  // namespace

void orc_soft_sgm_fwd(const double* C, int W, int H, int D, double p1, double p2, int paths,
                      double tau, double* S, double* dhat) {
    const size_t n = (size_t)W * H * D;
    std::memset(S, 0, n * sizeof(double));
    auto ws = soft_walks(W, H, paths);
    std::vector<double> Lb;
    for (const DWalk& w : ws) {
        soft_path_forward(C, W, D, p1, p2, w, Lb);
        int X = w.sx, Y = w.sy;
        for (int t = 0; t < w.len; t++, X += w.dx, Y += w.dy)
            for (int z = 0; z < D; z++) S[((size_t)Y * W + X) * D + z] += Lb[(size_t)t * D + z];
    }
    for (size_t p = 0; p < (size_t)W * H; p++) {
        const double* s = S + p * D;
        double mn = std::numeric_limits<double>::infinity();
        for (int z = 0; z < D; z++) mn = std::fmin(mn, s[z]);
        double den = 0, num = 0;
        for (int z = 0; z < D; z++) {
            const double e = std::exp(-(s[z] - mn) / tau);
            den += e; num += z * e;
        }
        dhat[p] = num / den;
    }
}

void orc_soft_sgm_bwd(const double* C, int W, int H, int D, double p1, double p2, int paths,
                      double tau, const double* g_dhat, double* dC, double* dP1, double* dP2) {
    const size_t n = (size_t)W * H * D;
    std::vector<double> S(n), dh((size_t)W * H), dS(n);
    orc_soft_sgm_fwd(C, W, H, D, p1, p2, paths, tau, S.data(), dh.data());
    for (size_t p = 0; p < (size_t)W * H; p++) {
        const double* s = &S[p * D];
        double mn = std::numeric_limits<double>::infinity();
        for (int z = 0; z < D; z++) mn = std::fmin(mn, s[z]);
        double den = 0;
        for (int z = 0; z < D; z++) den += std::exp(-(s[z] - mn) / tau);
        for (int z = 0; z < D; z++) {
            const double pz = std::exp(-(s[z] - mn) / tau) / den;
            dS[p * D + z] = g_dhat[p] * (-1.0 / tau) * pz * (z - dh[p]);
        }
    }
    std::memset(dC, 0, n * sizeof(double));
    double gp1 = 0, gp2 = 0;
    const double inf = std::numeric_limits<double>::infinity();
    auto ws = soft_walks(W, H, paths);
    std::vector<double> Lb, carry(D), G(D);
    for (const DWalk& w : ws) {
        soft_path_forward(C, W, D, p1, p2, w, Lb);
        std::fill(carry.begin(), carry.end(), 0.0);
        for (int t = w.len - 1; t >= 0; t--) {
            const int X = w.sx + t * w.dx, Y = w.sy + t * w.dy;
            const size_t po = ((size_t)Y * W + X) * D;
            for (int z = 0; z < D; z++) {
                G[z] = dS[po + z] + carry[z];
                dC[po + z] += G[z];
            }
            if (t == 0) break;
            const double* Lp = &Lb[(size_t)(t - 1) * D];
            double m = inf;
            int ks = 0;
            for (int z = 0; z < D; z++) if (Lp[z] < m) { m = Lp[z]; ks = z; }
            std::fill(carry.begin(), carry.end(), 0.0);
            double gm = 0;
            for (int z = 0; z < D; z++) {
                const double a = Lp[z];
                const double b = z > 0 ? Lp[z - 1] + p1 : inf;
                const double e = z < D - 1 ? Lp[z + 1] + p1 : inf;
                const double f = m + p2;
                const double mn = std::fmin(a, std::fmin(b, std::fmin(e, f)));
                const double gz = G[z];
                if (a == mn) carry[z] += gz;
                else if (b == mn) { carry[z - 1] += gz; gp1 += gz; }
                else if (e == mn) { carry[z + 1] += gz; gp1 += gz; }
                else { gm += gz; gp2 += gz; }
                gm -= gz;
            }
            carry[ks] += gm;
        }
    }
    *dP1 = gp1;
    *dP2 = gp2;
}

}  // extern "C"
