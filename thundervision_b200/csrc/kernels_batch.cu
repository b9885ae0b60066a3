// Batched fused stereo: many integer-domain pairs of uneven size and
// disparity range aggregated by ONE persistent launch.
//
// Work queue.  Every pass of every pair is cut into work items -- a band of
// rows for the BT-plane prep, a group of G path lines for a vertical or
// diagonal pass, a group of rows for a horizontal pass -- and the items are
// laid out pass-major (all pairs' prep, then all pairs' V+, ...), pairs in a
// fixed order inside each pass.  The grid is one block per SM; each block
// takes the next item with one atomicAdd on the queue head and runs the same
// device body the per-frame kernels run (fused_body.cuh).  Passes of one pair
// read-modify-write the same aggregation volume, so an item waits until every
// item of its pair's previous pass has completed: per (pair, pass) a counter
// is incremented (release) after an item's block barrier, and the waiting
// block polls it (acquire).  Items are handed out in queue order, so the
// items a block waits for were taken earlier by blocks that are already
// running and never wait on later items: the queue cannot deadlock.
//
// Every wait is bounded.  A dependency wait that runs out records
// TDV_ERR_TIMEOUT; an item whose pair, pass or block index is out of range
// records TDV_ERR_BAD_WORK without touching memory; once the error word is
// set every block stops taking items.  The queue lives in device memory and
// the whole launch (one memset of the control words + the kernel) is what a
// CUDA graph captures for video streams.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "fused_body.cuh"

namespace tdv {

namespace {

constexpr int kPasses = 9;  // prep, V+, V-, D1+, D1-, D2+, D2-, H+, H-(WTA)
constexpr int kBatchWarps = kMaxG + 1;  // one block per SM
constexpr int kBatchWarps2 = 13;        // two blocks per SM
constexpr int kSmemBudget2 = 110 * 1024;  // dynamic shared memory per block at two per SM
constexpr int kPrepPixels = 16384;  // pixels per prep item
constexpr int kCtlHeader = 4;       // ints: queue head, error word, 2 spare

struct BPair {
    FK k;
    ImgArg L, R;
    int ppl, G, hrows, hsplit, hwb, hrb, prep_rows, pad;
    int nb[kPasses];   // items per pass (0: pass not run)
    int dep[kPasses];  // pass this pass waits for, -1 none
};

struct BItem {
    int32_t pp;   // pair * 16 + pass
    int32_t blk;  // block index inside the pass
};

// walk direction of each pass (the order of the per-frame launches)
__constant__ signed char kPassDx[kPasses] = {0, 0, 0, 1, -1, -1, 1, 1, -1};
__constant__ signed char kPassDy[kPasses] = {0, 1, -1, 1, -1, 1, -1, 0, 0};
constexpr signed char kPassDxHost[kPasses] = {0, 0, 0, 1, -1, -1, 1, 1, -1};
constexpr signed char kPassDyHost[kPasses] = {0, 1, -1, 1, -1, 1, -1, 0, 0};

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_volatile(const int* p) { return *(const volatile int*)p; }
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Waits until *cnt >= target; false on timeout (recorded) or on an error
// recorded by another block.
__device__ bool wait_done(const int* cnt, int target, int* err, uint64_t limit_ns) {
    if (ld_acquire(cnt) >= target) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        __nanosleep(200);
        if (ld_acquire(cnt) >= target) return true;
        if (ld_volatile(err) != 0) return false;
        if (global_ns() - t0 > limit_ns) {
            atomicCAS(err, 0, (int)TDV_ERR_TIMEOUT);
            return false;
        }
    }
}

template <int MODE, bool DIAG>
__device__ __forceinline__ void run_vd(const BPair& P, int pass, int blk, unsigned char* smem) {
    const FK& k = P.k;
    const int dx = kPassDx[pass], dy = kPassDy[pass], s = dx * dy;
    const int nlines = s == 0 ? k.W : k.W + k.H - 1;
    const int kmin = s > 0 ? -(k.H - 1) : 0;
    if (P.ppl == 1) vd_body<1, MODE, DIAG>(k, s, dy, kmin, nlines, P.G, blk, smem);
    else if (P.ppl == 2) vd_body<2, MODE, DIAG>(k, s, dy, kmin, nlines, P.G, blk, smem);
    else vd_body<4, MODE, DIAG>(k, s, dy, kmin, nlines, P.G, blk, smem);
}

template <int MODE>
__device__ __forceinline__ void run_h(const BPair& P, int dx, int blk, unsigned char* smem) {
    const FK& k = P.k;
    if (P.hsplit) {
        if (P.ppl == 2) h2_body<1, MODE>(k, dx, P.hrows, P.hwb, P.hrb, blk, smem, false);
        else h2_body<2, MODE>(k, dx, P.hrows, P.hwb, P.hrb, blk, smem, false);
    } else {
        if (P.ppl == 1) hp_body<1, MODE, false>(k, dx, P.hrows, blk, smem);
        else if (P.ppl == 2) hp_body<2, MODE, false>(k, dx, P.hrows, blk, smem);
        else hp_body<4, MODE, false>(k, dx, P.hrows, blk, smem);
    }
}

// NW warps per block: one 800-thread block per SM (NW = 25) or two 416-thread
// blocks per SM (NW = 13), each taking its own work items
template <int NW>
__global__ void __launch_bounds__(NW * 32, NW == kBatchWarps ? 1 : 2)
    batch_kernel(const BPair* __restrict__ pairs, int npairs, const BItem* __restrict__ items, int nitems,
                 int* ctl, unsigned long long wait_ns, unsigned long long* trace) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ BPair sp;
    __shared__ int s_pass, s_blk, s_stop, s_slot, s_item, s_pp;
    __shared__ unsigned long long s_take, s_go;
    int* head = ctl;
    int* err = ctl + 1;
    int* done = ctl + kCtlHeader;

    for (;;) {
        if (threadIdx.x == 0) {
            int stop = 1;
            if (ld_volatile(err) == 0) {
                const int i = atomicAdd(head, 1);
                s_item = i;
                if (trace) s_take = global_ns();
                if (i < nitems) {
                    const BItem it = items[i];
                    s_pp = it.pp;
                    const unsigned pair = (unsigned)it.pp >> 4;
                    const int pass = it.pp & 15;
                    if (pair >= (unsigned)npairs || pass >= kPasses || it.blk < 0 ||
                        it.blk >= pairs[pair].nb[pass]) {
                        atomicCAS(err, 0, (int)TDV_ERR_BAD_WORK);
                    } else {
                        const int dp = pairs[pair].dep[pass];
                        if (dp < 0 || wait_done(done + pair * kPasses + dp, pairs[pair].nb[dp], err, wait_ns)) {
                            stop = 0;
                            sp = pairs[pair];
                            s_pass = pass;
                            s_blk = it.blk;
                            s_slot = pair * kPasses + pass;
                            if (trace) s_go = global_ns();
                        }
                    }
                }
            }
            s_stop = stop;
        }
        __syncthreads();
        if (s_stop) break;
        // data of the previous pass was published by generic stores of other
        // blocks; this block reads it through TMA (async proxy)
        fence_proxy_async_global();
        const int pass = s_pass, blk = s_blk;
        if (pass == 0) {
            const FK& k = sp.k;
            const int y0 = blk * sp.prep_rows, y1 = min(k.H, y0 + sp.prep_rows);
            const int n = (y1 - y0) * k.W;
            Plane* LP = const_cast<Plane*>(k.LP);
            Plane* RPp = const_cast<Plane*>(k.RPp);
            for (int i = threadIdx.x; i < n; i += blockDim.x)
                prep_pixel(sp.L, sp.R, LP, RPp, k.W, k.Wp, i % k.W, y0 + i / k.W);
        } else if (pass == 1) {
            run_vd<0, false>(sp, pass, blk, smem);
        } else if (pass == 2) {
            run_vd<1, false>(sp, pass, blk, smem);
        } else if (pass <= 6) {
            run_vd<1, true>(sp, pass, blk, smem);
        } else if (pass == 7) {
            run_h<1>(sp, 1, blk, smem);
        } else {
            run_h<2>(sp, -1, blk, smem);
        }
        // generic shared-memory accesses of this item before the next item's
        // TMA writes into the same bytes
        fence_proxy_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_proxy_async_global();
            __threadfence();
            atomicAdd(done + s_slot, 1);
            if (trace) {
                // diagnostic: when the item was taken, when its dependency was
                // met, when it ended, the SM it ran on and its pair * 16 + pass
                unsigned smid;
                asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
                unsigned long long* t = trace + 4 * (size_t)s_item;
                t[0] = s_take;
                t[1] = s_go;
                t[2] = global_ns();
                t[3] = ((unsigned long long)smid << 32) | (unsigned)s_pp;
            }
        }
    }
}

// ------------------------------------------------------------- host side
size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Estimated relative duration of one item of `pass` (sorting key): the
// serial chain length times the per-step work.
double item_weight(const BatchPairArgs& p, int pass) {
    const int ppl = ppl_for(p.D);
    if (pass == 0) return (double)p.W * p.H / kPrepPixels;
    if (pass <= 6) return (double)p.H * (1 + ppl);
    return (double)p.W * (1 + ppl);
}

}  // namespace

int batch_passes() { return kPasses; }
int batch_threads() { return kBatchWarps * 32; }
size_t batch_ctl_bytes(int npairs) { return sizeof(int) * (kCtlHeader + (size_t)kPasses * npairs); }

size_t batch_scratch_bytes(const std::vector<BatchPairArgs>& pairs) {
    size_t b = 0;
    for (const auto& p : pairs) b += align256(fused_plane_bytes(p.W, p.H)) + align256(fused_agg_bytes(p.W, p.H, p.D));
    return b;
}

const char* batch_plan(const std::vector<BatchPairArgs>& pairs, int p1h, int p2h, int paths,
                       const BatchTiles& t, unsigned char* scratch, unsigned char* d_desc, BatchPlan& out) {
    const int n = (int)pairs.size();
    if (t.lines_per_cta < 1 || t.lines_per_cta > kMaxG) return "lines_per_cta must be in [1, 24]";
    if (t.rows_per_cta < 1 || t.rows_per_cta > kBatchWarps) return "rows_per_cta must be in [1, 25]";
    if (t.ctas_per_sm != 1 && t.ctas_per_sm != 2) return "ctas_per_sm must be 1 or 2";
    const int NW = t.ctas_per_sm == 2 ? kBatchWarps2 : kBatchWarps;
    const int budget = t.ctas_per_sm == 2 ? kSmemBudget2 : kSmemBudget;
    std::vector<BPair> hp(n);
    out.ctl_off = 0;
    int smem = 0;
    size_t off = 0;
    const uint32_t big = 511u + 2u * (uint32_t)p2h;
    for (int i = 0; i < n; i++) {
        const BatchPairArgs& a = pairs[i];
        BPair& P = hp[i];
        memset(&P, 0, sizeof(P));
        FK& k = P.k;
        Plane* LP = (Plane*)(scratch + off);
        off += align256(fused_plane_bytes(a.W, a.H));
        k.LP = LP;
        k.RPp = LP + (size_t)a.W * a.H;
        k.S = (uint32_t*)(scratch + off);
        off += align256(fused_agg_bytes(a.W, a.H, a.D));
        k.W = a.W;
        k.H = a.H;
        k.D = a.D;
        k.Wp = padded_len(a.W);
        P.ppl = ppl_for(a.D);
        k.Dp2 = 32 * P.ppl;
        k.P1P1 = (uint32_t)p1h * 0x10001u;
        k.P2P2 = (uint32_t)p2h * 0x10001u;
        k.BIGBIG = big * 0x10001u;
        k.disp = a.disp;
        k.disp_norm = a.disp_norm;
        k.disp_right = a.disp_right;
        k.lr_thr = a.lr_thr;
        k.err = (int*)(d_desc + out.ctl_off) + 1;
        k.S2 = nullptr;
        P.L = a.L;
        P.R = a.R;

        // vertical / diagonal: G lines per item
        int G = std::min(std::min(t.lines_per_cta, NW - 1), std::max(a.W, 1));
        while (G > 1 && vd_smem_bytes(G, P.ppl) > budget) G--;
        if (vd_smem_bytes(G, P.ppl) > budget) return "vertical pass tile does not fit in shared memory";
        P.G = G;
        smem = std::max(smem, vd_smem_bytes(G, P.ppl));
        // horizontal: rows per item; the L-R rows only in the last pass
        const bool lr = a.lr_thr >= 0;
        P.hsplit = (P.ppl >= 2 && t.split_disparity) ? 1 : 0;
        int rows = t.rows_per_cta;
        if (P.hsplit) {
            const int ph = P.ppl / 2;
            rows = std::min(rows, std::min(NW / 2, kMaxRowsH2 * 2 - 1));
            P.hwb = h2_warp_bytes(ph);
            P.hrb = h2_row_bytes(lr, a.W);
            while (rows > 1 && rows * (2 * P.hwb + P.hrb) > budget) rows--;
            if (rows * (2 * P.hwb + P.hrb) > budget) return "horizontal pass tile does not fit in shared memory";
            smem = std::max(smem, rows * (2 * P.hwb + P.hrb));
        } else {
            // producer-fed rows: one consumer warp per row plus the producer warp
            rows = std::min(rows, NW - 1);
            while (rows > 1 && hp_smem_bytes(rows, P.ppl, lr, a.W, false) > budget) rows--;
            if (hp_smem_bytes(rows, P.ppl, lr, a.W, false) > budget)
                return "horizontal pass tile does not fit in shared memory";
            smem = std::max(smem, hp_smem_bytes(rows, P.ppl, lr, a.W, false));
        }
        P.hrows = rows;
        P.prep_rows = std::max(1, kPrepPixels / a.W);

        const int order8[kPasses] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
        const int order4[5] = {0, 1, 2, 7, 8};
        const int* ord = paths == 8 ? order8 : order4;
        const int np = paths == 8 ? kPasses : 5;
        for (int p = 0; p < kPasses; p++) {
            P.nb[p] = 0;
            P.dep[p] = -1;
        }
        for (int j = 0; j < np; j++) {
            const int p = ord[j];
            int nb;
            if (p == 0) {
                nb = (a.H + P.prep_rows - 1) / P.prep_rows;
            } else if (p <= 6) {
                const int s = kPassDxHost[p] * kPassDyHost[p];
                const int nlines = s == 0 ? a.W : a.W + a.H - 1;
                nb = (nlines + G - 1) / G;
            } else {
                nb = (a.H + rows - 1) / rows;
            }
            P.nb[p] = nb;
            P.dep[p] = j == 0 ? -1 : ord[j - 1];
        }
    }

    // queue: pass-major; inside a pass, pairs by decreasing item weight (or
    // in input order)
    std::vector<BItem> items;
    const int passes8[kPasses] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
    for (int p : passes8) {
        std::vector<int> idx(n);
        std::iota(idx.begin(), idx.end(), 0);
        if (t.order == TDV_BATCH_ORDER_LONGEST_FIRST)
            std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
                return item_weight(pairs[a], p) > item_weight(pairs[b], p);
            });
        for (int i : idx) {
            // a pair's diagonal line groups span 1..H rows: longest first
            std::vector<int> blks(hp[i].nb[p]);
            std::iota(blks.begin(), blks.end(), 0);
            if (p >= 3 && p <= 6 && t.order == TDV_BATCH_ORDER_LONGEST_FIRST) {
                const BatchPairArgs& a = pairs[i];
                const int s = kPassDxHost[p] * kPassDyHost[p];
                const int nlines = a.W + a.H - 1, kmin = s > 0 ? -(a.H - 1) : 0, G = hp[i].G;
                std::vector<int> rows(blks.size());
                for (size_t j = 0; j < blks.size(); j++)
                    rows[j] = group_rows(a.W, a.H, s, kmin + (int)j * G, std::min(G, nlines - (int)j * G));
                std::stable_sort(blks.begin(), blks.end(), [&](int x, int y) { return rows[x] > rows[y]; });
            }
            for (int b : blks) items.push_back(BItem{i * 16 + p, b});
        }
    }

    out.n_pairs = n;
    out.n_items = (int)items.size();
    out.smem = smem;
    out.ctas_per_sm = t.ctas_per_sm;
    out.pairs_off = align256(batch_ctl_bytes(n));
    out.items_off = out.pairs_off + align256(sizeof(BPair) * n);
    out.bytes = out.items_off + sizeof(BItem) * items.size();
    out.item_bytes = (int)sizeof(BItem);
    out.desc.assign(out.bytes, 0);
    memcpy(out.desc.data() + out.pairs_off, hp.data(), sizeof(BPair) * n);
    memcpy(out.desc.data() + out.items_off, items.data(), sizeof(BItem) * items.size());
    return nullptr;
}

template <int NW>
cudaError_t configure_nw(const BatchPlan& plan) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, batch_kernel<NW>);
    if (e != cudaSuccess) return e;
    if (fa.maxThreadsPerBlock < NW * 32) return cudaErrorInvalidConfiguration;
    return cudaFuncSetAttribute(batch_kernel<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, plan.smem);
}

cudaError_t batch_configure(const BatchPlan& plan) {
    return plan.ctas_per_sm == 2 ? configure_nw<kBatchWarps2>(plan) : configure_nw<kBatchWarps>(plan);
}

cudaError_t batch_launch(const BatchPlan& plan, unsigned char* d_desc, unsigned long long wait_ns, int grid,
                         cudaStream_t st, unsigned long long* trace) {
    cudaError_t e = cudaMemsetAsync(d_desc + plan.ctl_off, 0, batch_ctl_bytes(plan.n_pairs), st);
    if (e != cudaSuccess) return e;
    const BPair* pairs = (const BPair*)(d_desc + plan.pairs_off);
    const BItem* items = (const BItem*)(d_desc + plan.items_off);
    int* ctl = (int*)(d_desc + plan.ctl_off);
    if (plan.ctas_per_sm == 2)
        batch_kernel<kBatchWarps2><<<2 * grid, kBatchWarps2 * 32, plan.smem, st>>>(pairs, plan.n_pairs, items,
                                                                                   plan.n_items, ctl, wait_ns, trace);
    else
        batch_kernel<kBatchWarps><<<grid, kBatchWarps * 32, plan.smem, st>>>(pairs, plan.n_pairs, items,
                                                                             plan.n_items, ctl, wait_ns, trace);
    return cudaGetLastError();
}

}  // namespace tdv
