// Per-frame launches of the fused integer-domain path: one kernel per pass
// (prep, V+, V-, D1+, D1-, D2+, D2-, H+, H- with WTA), each a thin wrapper
// around the device bodies in fused_body.cuh.
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "fused_body.cuh"

namespace tdv {

namespace {

__global__ void prep_kernel(ImgArg L, ImgArg R, Plane* LP, Plane* RPp, int W, int H, int Wp) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < W) prep_pixel(L, R, LP, RPp, W, Wp, x, blockIdx.y);
}

// Diagonal passes: a line group's row count ramps from 1 to H across the
// image corners, so groups are paired (a short one after a long one) into
// blocks of about H rows each; the table travels as a kernel parameter.
constexpr int kMaxPairedBlocks = 256;
struct GroupPairs {
    int16_t first[kMaxPairedBlocks];
    int16_t second[kMaxPairedBlocks];  // -1: none
};

// Lines per block, vertical/diagonal passes: at most 15 consumer warps and the
// producer, so that two blocks (one of each concurrent pass chain) share an SM.
constexpr int kVdMaxG = 15;

template <int PPL, int MODE, bool DIAG, int VAR>
__global__ void __launch_bounds__((kVdMaxG + 1) * 32, 2)
    vd_pass(FK k, int s, int dy, int kmin, int nlines, int G, GroupPairs gp, int paired) {
    extern __shared__ __align__(128) unsigned char smem[];
    if (!paired) {
        vd_body<PPL, MODE, DIAG, VAR>(k, s, dy, kmin, nlines, G, blockIdx.x, smem);
        return;
    }
    vd_body<PPL, MODE, DIAG, VAR>(k, s, dy, kmin, nlines, G, gp.first[blockIdx.x], smem);
    const int j2 = gp.second[blockIdx.x];
    if (j2 >= 0) vd_body<PPL, MODE, DIAG, VAR>(k, s, dy, kmin, nlines, G, j2, smem);
}

constexpr int kHpMaxRows = 16;  // consumer warps per block, horizontal passes
// Registers per thread of the horizontal passes: 112 keeps the last pass's
// keys and register window off the stack, and still leaves room on an SM for
// one vertical/diagonal block (512 threads x 64 registers) beside a
// horizontal block of up to 9 warps (a full-HD frame's 8 rows per block), so
// the next frame's passes can overlap this frame's last pass; a block of
// kHpMaxRows + 1 warps (17 x 32 x 112 registers) still fits an SM.
constexpr int kHpRegs = 112;
static_assert((kHpMaxRows + 1) * 32 * kHpRegs <= 65536, "a horizontal block must fit the register file");

template <int PPL, int MODE, bool TWO, int VAR>
__global__ void __maxnreg__(kHpRegs) hp_pass(FK k, int dx, int R) {
    extern __shared__ __align__(128) unsigned char smem[];
    hp_body<PPL, MODE, TWO, VAR>(k, dx, R, blockIdx.x, smem);
}

// The last pass runs alone at the end of a frame: under the reference
// weights (VAR > 0) its keys, border flags and repeated-cell columns stay in
// registers at 168 per thread (measured on a full-HD frame, D = 256: 0.58 ms
// against 0.64 ms at 112); the standard variant needs no more than 112 and
// keeps room for the next frame's first pass beside it.
constexpr int hp_wta_regs(int var) { return var == 0 ? kHpRegs : 168; }
constexpr int hp_wta_max_rows(int var) {
    return 65536 / (32 * hp_wta_regs(var)) - 1 < kHpMaxRows ? 65536 / (32 * hp_wta_regs(var)) - 1 : kHpMaxRows;
}
template <int PPL, bool TWO, int VAR>
__global__ void __maxnreg__(hp_wta_regs(VAR)) hp_wta_pass(FK k, int dx, int R) {
    extern __shared__ __align__(128) unsigned char smem[];
    hp_body<PPL, 2, TWO, VAR>(k, dx, R, blockIdx.x, smem);
}

// ------------------------------------------------------------- host side
int sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

// Opts a kernel into `bytes` of dynamic shared memory on the current device,
// once: later launches needing no more skip the driver call.
cudaError_t opt_in_smem(const void* fn, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    int& cur = done[{fn, dev}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

// Greedy pairing: groups by decreasing row count, each block takes the
// longest left and, if it fits under the longest, the shortest left.
// Returns the block count, or -1 if the table would overflow.
int pair_groups(int W, int H, int s, int kmin, int nlines, int G, GroupPairs& gp) {
    const int ng = (nlines + G - 1) / G;
    if (ng > 2 * kMaxPairedBlocks) return -1;
    std::vector<int> rows(ng), order(ng);
    for (int j = 0; j < ng; j++) {
        rows[j] = group_rows(W, H, s, kmin + j * G, std::min(G, nlines - j * G));
        order[j] = j;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return rows[a] > rows[b]; });
    for (int b = 0; b < kMaxPairedBlocks; b++) gp.first[b] = gp.second[b] = -1;
    const int cap = rows[order[0]];
    int lo = 0, hi = ng - 1, nb = 0;
    while (lo <= hi) {
        if (nb >= kMaxPairedBlocks) return -1;
        const int j = order[lo++];
        gp.first[nb] = (int16_t)j;
        gp.second[nb] = -1;
        if (lo <= hi && rows[j] + rows[order[hi]] <= cap) gp.second[nb] = (int16_t)order[hi--];
        nb++;
    }
    return nb;
}

int pair_count(const GroupPairs& gp) {
    int n = 0;
    while (n < kMaxPairedBlocks && gp.first[n] >= 0) n++;
    return n;
}

template <int PPL, int MODE, bool DIAG, int VAR>
cudaError_t launch_vd(const FK& k, int dx, int dy, cudaStream_t st) {
    const int s = dx * dy;
    const int nlines = s == 0 ? k.W : k.W + k.H - 1;
    const int kmin = s > 0 ? -(k.H - 1) : 0;
    const int nsm = sm_count();
    GroupPairs gp;
    int paired = 0, blocks = 0;
    int G = (k.W + nsm - 1) / nsm;
    G = G < 1 ? 1 : (G > kVdMaxG ? kVdMaxG : G);
    if (DIAG) {
        // smallest G whose paired blocks fit one wave (cached per shape)
        static std::mutex mu;
        static std::map<std::tuple<int, int, int, int>, std::pair<int, GroupPairs>> cache;
        const auto key = std::make_tuple(k.W, k.H, s, nsm);
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it == cache.end()) {
            int g = G, nb = -1;
            for (; g <= kVdMaxG; g++) {
                nb = pair_groups(k.W, k.H, s, kmin, nlines, g, gp);
                if (nb > 0 && nb <= nsm) break;
            }
            if (g > kVdMaxG) {
                g = kVdMaxG;
                nb = pair_groups(k.W, k.H, s, kmin, nlines, g, gp);
            }
            if (cache.size() > 64) cache.clear();
            it = cache.emplace(key, std::make_pair(nb > 0 ? g : -g, gp)).first;
        }
        G = it->second.first > 0 ? it->second.first : -it->second.first;
        paired = it->second.first > 0;
        gp = it->second.second;
        blocks = paired ? pair_count(gp) : 0;
    }
    if (!paired) blocks = (nlines + G - 1) / G;
    const int smem = vd_smem_bytes(G, PPL);
    if (smem > kSmemBudget) return cudaErrorInvalidConfiguration;
    cudaError_t e = opt_in_smem((const void*)vd_pass<PPL, MODE, DIAG, VAR>, smem);
    if (e != cudaSuccess) return e;
    vd_pass<PPL, MODE, DIAG, VAR><<<blocks, (G + 1) * 32, smem, st>>>(k, s, dy, kmin, nlines, G, gp, paired);
    return cudaGetLastError();
}

// rows per block: spread the rows over every SM, at most max_rows (a pass
// that shares the SMs with a concurrent chain keeps its blocks small)
template <int PPL, int MODE, bool TWO, int VAR>
cudaError_t launch_hp(const FK& k, int dx, int max_rows, cudaStream_t st) {
    const bool lr = MODE == 2 && k.lr_thr >= 0;
    const int nsm = sm_count();
    int R = (k.H + nsm - 1) / nsm;
    const int cap = MODE == 2 ? hp_wta_max_rows(VAR) : kHpMaxRows;
    if (max_rows > cap) max_rows = cap;
    R = R < 1 ? 1 : (R > max_rows ? max_rows : R);
    while (R > 1 && hp_smem_bytes(R, PPL, lr, k.W, TWO) > kSmemBudget) R--;
    const int smem = hp_smem_bytes(R, PPL, lr, k.W, TWO);
    if (smem > kSmemBudget) return cudaErrorInvalidConfiguration;
    const int blocks = (k.H + R - 1) / R;
    if constexpr (MODE == 2) {
        cudaError_t e = opt_in_smem((const void*)hp_wta_pass<PPL, TWO, VAR>, smem);
        if (e != cudaSuccess) return e;
        hp_wta_pass<PPL, TWO, VAR><<<blocks, (R + 1) * 32, smem, st>>>(k, dx, R);
    } else {
        cudaError_t e = opt_in_smem((const void*)hp_pass<PPL, MODE, TWO, VAR>, smem);
        if (e != cudaSuccess) return e;
        hp_pass<PPL, MODE, TWO, VAR><<<blocks, (R + 1) * 32, smem, st>>>(k, dx, R);
    }
    return cudaGetLastError();
}

// The FK of one pass: its direction's weight classes and side rows
// (fused direction order V+ V- D1+ D1- D2+ D2- H+ H-).
FK for_dir(const FK& base, const FusedArgs& a, int dir) {
    FK r = base;
    const FusedWeights* fw = a.fw;
    if (!fw || !a.weights) return r;
    if (fw->has_line) r.lw = a.weights + fw->lw_off + (size_t)dir * fw->nl;
    if (fw->has_border) r.bw = a.weights + fw->bw_off + (size_t)dir * fw->nb;
    if (fw->has_corner && (dir == 3 || dir == 5)) r.side = a.side + (size_t)(dir == 3 ? 0 : 1) * a.H * base.Dp2;
    if (fw->has_corner && dir == 7) {
        r.corner = (const int*)(a.weights + fw->corner_off);
        r.side_all = a.side;
    }
    return r;
}

template <int PPL, int VAR>
cudaError_t run_fused(const FK& k, const FusedArgs& a, cudaStream_t st, Timer* tm) {
    cudaError_t e;
    auto mark = [&](const char* n, cudaStream_t s) {
        if (tm) tm->mark_on(n, s);
    };
    const FK kv1 = for_dir(k, a, 0), kv2 = for_dir(k, a, 1), kd1 = for_dir(k, a, 2), kd2 = for_dir(k, a, 3),
             kd3 = for_dir(k, a, 4), kd4 = for_dir(k, a, 5), kh1 = for_dir(k, a, 6), kh2 = for_dir(k, a, 7);
    const bool chains = a.paths == 8 && a.agg2 && a.side_stream && a.fork && a.join;
    if (!chains) {
        if ((e = launch_vd<PPL, 0, false, VAR>(kv1, 0, 1, st)) != cudaSuccess) return e;
        mark("fused_pass_V+", st);
        if ((e = launch_vd<PPL, 1, false, VAR>(kv2, 0, -1, st)) != cudaSuccess) return e;
        mark("fused_pass_V-", st);
        if (a.paths == 8) {
            if ((e = launch_vd<PPL, 1, true, VAR>(kd1, 1, 1, st)) != cudaSuccess) return e;
            mark("fused_pass_D1+", st);
            if ((e = launch_vd<PPL, 1, true, VAR>(kd2, -1, -1, st)) != cudaSuccess) return e;
            mark("fused_pass_D1-", st);
            if ((e = launch_vd<PPL, 1, true, VAR>(kd3, -1, 1, st)) != cudaSuccess) return e;
            mark("fused_pass_D2+", st);
            if ((e = launch_vd<PPL, 1, true, VAR>(kd4, 1, -1, st)) != cudaSuccess) return e;
            mark("fused_pass_D2-", st);
        }
        if ((e = launch_hp<PPL, 1, false, VAR>(kh1, 1, kMaxG, st)) != cudaSuccess) return e;
        mark("fused_pass_H+", st);
        if ((e = launch_hp<PPL, 2, false, VAR>(kh2, -1, kMaxG, st)) != cudaSuccess) return e;
        mark("fused_pass_H-_wta", st);
        return cudaSuccess;
    }
    // two chains: V+ V- D1+ into S on the call's stream, D1- D2+ D2- into S2
    // on the side stream (V+ and D1- store their volume, the first touch);
    // then H+ joins them (S += S2 + L) and H- finishes S
    // With per-kernel timing on, the chains run one after the other on the
    // call's stream (same kernels, same volumes) so that each kernel's
    // events time it alone.
    const bool concurrent = !(tm && tm->on);
    cudaStream_t sd = concurrent ? a.side_stream : st;
    FK kb2 = kd2, kb3 = kd3, kb4 = kd4;
    kb2.S = kb3.S = kb4.S = (uint32_t*)a.agg2;
    if (concurrent) {
        if ((e = cudaEventRecord(a.fork, st)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(sd, a.fork, 0)) != cudaSuccess) return e;
        if (tm) tm->fork(sd);
    }
    if ((e = launch_vd<PPL, 0, true, VAR>(kb2, -1, -1, sd)) != cudaSuccess) return e;
    mark("fused_pass_D1-", sd);
    if ((e = launch_vd<PPL, 0, false, VAR>(kv1, 0, 1, st)) != cudaSuccess) return e;
    mark("fused_pass_V+", st);
    if ((e = launch_vd<PPL, 1, true, VAR>(kb3, -1, 1, sd)) != cudaSuccess) return e;
    mark("fused_pass_D2+", sd);
    if ((e = launch_vd<PPL, 1, false, VAR>(kv2, 0, -1, st)) != cudaSuccess) return e;
    mark("fused_pass_V-", st);
    if ((e = launch_vd<PPL, 1, true, VAR>(kb4, 1, -1, sd)) != cudaSuccess) return e;
    mark("fused_pass_D2-", sd);
    if ((e = launch_vd<PPL, 1, true, VAR>(kd1, 1, 1, st)) != cudaSuccess) return e;
    mark("fused_pass_D1+", st);
    if (concurrent) {
        if ((e = cudaEventRecord(a.join, sd)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(st, a.join, 0)) != cudaSuccess) return e;
        if (tm) tm->join();
    }
    FK kj = kh1;
    kj.S2 = (const uint32_t*)a.agg2;
    if ((e = launch_hp<PPL, 1, true, VAR>(kj, 1, kMaxG, st)) != cudaSuccess) return e;
    mark("fused_pass_H+", st);
    if ((e = launch_hp<PPL, 2, false, VAR>(kh2, -1, kMaxG, st)) != cudaSuccess) return e;
    mark("fused_pass_H-_wta", st);
    return cudaSuccess;
}

}  // namespace

size_t fused_plane_bytes(int W, int H) {
    return ((size_t)W * H + (size_t)padded_len(W) * H) * sizeof(Plane);
}

size_t fused_agg_bytes(int W, int H, int D) {
    return (size_t)W * H * 64 * ppl_for(D) * sizeof(uint16_t);
}

cudaError_t launch_fused(const FusedArgs& a, cudaStream_t st, Timer* tm) {
    Plane* LP = (Plane*)a.planes;
    Plane* RPp = LP + (size_t)a.W * a.H;
    const int Wp = padded_len(a.W);
    dim3 pb(128), pg((a.W + 127) / 128, a.H);
    prep_kernel<<<pg, pb, 0, st>>>(a.L, a.R, LP, RPp, a.W, a.H, Wp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (tm) tm->mark("fused_prep");
    FK k;
    k.LP = LP;
    k.RPp = RPp;
    k.S = (uint32_t*)a.agg;
    k.W = a.W;
    k.H = a.H;
    k.D = a.D;
    k.Wp = Wp;
    const int ppl = ppl_for(a.D);
    k.Dp2 = 32 * ppl;
    const uint32_t big = (uint32_t)a.off_h + 511u + 2u * (uint32_t)a.p2h;
    k.P1P1 = (uint32_t)a.p1h * 0x10001u;
    k.P2P2 = (uint32_t)a.p2h * 0x10001u;
    k.BIGBIG = big * 0x10001u;
    k.OFFOFF = (uint32_t)a.off_h * 0x10001u;
    k.lw = nullptr;
    k.bw = nullptr;
    k.side = nullptr;
    k.corner = nullptr;
    k.side_all = nullptr;
    k.GSTART = (uint32_t)a.gstart * 0x10001u;
    k.disp = a.disp;
    k.disp_norm = a.disp_norm;
    k.disp_right = a.disp_right;
    k.lr_thr = a.lr_thr;
    k.err = a.err;
    k.S2 = nullptr;
    // kernel variant: 0 the STANDARD recurrence over the full table (none of
    // the reference-weight code compiled in); else 1, with the excluded
    // minimum of the reference CPU recurrence 2 (D-1 is the high half of lane
    // 31's last pair: D fills the warp's span) or 3 (anywhere)
    const bool wtd = a.excl || a.gstart || a.off_h || (a.fw && a.weights);
    const int var = !wtd ? 0 : (!a.excl ? 1 : (a.D == 64 * ppl ? 2 : 3));
    switch (var * 4 + ppl) {
        case 1: return run_fused<1, 0>(k, a, st, tm);
        case 2: return run_fused<2, 0>(k, a, st, tm);
        case 4: return run_fused<4, 0>(k, a, st, tm);
        case 5: return run_fused<1, 1>(k, a, st, tm);
        case 6: return run_fused<2, 1>(k, a, st, tm);
        case 8: return run_fused<4, 1>(k, a, st, tm);
        case 9: return run_fused<1, 2>(k, a, st, tm);
        case 10: return run_fused<2, 2>(k, a, st, tm);
        case 12: return run_fused<4, 2>(k, a, st, tm);
        case 13: return run_fused<1, 3>(k, a, st, tm);
        case 14: return run_fused<2, 3>(k, a, st, tm);
        default: return run_fused<4, 3>(k, a, st, tm);
    }
}

}  // namespace tdv
