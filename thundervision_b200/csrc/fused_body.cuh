// Fused Birchfield-Tomasi + SGM + WTA (+ left-right check) for integer-domain
// inputs: u8 intensities used unscaled, P1/P2 multiples of 1/2, constant P2,
// D <= 256; the STANDARD recurrence over the FULL path table, or the
// reference's own CPU recurrence and path table (see "Reference semantics").
//
// Exactness.  In this domain every BT cost is a multiple of 1/2 in [0, 255]
// and every path cost L = C + min(...) - m' lies in [0, 255 + P2], so all
// quantities are small multiples of 1/2.  The kernels carry them as unsigned
// 16-bit "half-units" (2x the value), two disparities per 32-bit register.
// Integer arithmetic on these is exact, so the result is bit-identical to the
// float32 recurrence of the reference (tdvision/semiglobalcpu.cpp:104-122)
// evaluated on the same values, in any summation order.  Cells with x-d < 0
// (+INF in the reference) carry a sentinel BIG = 511 + 2*P2h that can never
// win a minimum and stays bounded: every invalid L is in [BIG, BIG + P2h] and
// every invalid S in [8*BIG, 8*(BIG + P2h)] <= 65535, above any valid S.
//
// Data flow per frame (8 paths):
//   prep : BT planes of both images (I, half-sample min, half-sample max in
//          half-units).  The right plane stores, at pixel x, the values of x
//          and x-1 so the disparity pair (d, d+1) of left column x reads one
//          16-byte entry; rows are padded with one 16-byte slot after every 8
//          entries so that lanes reading entries 8 apart hit distinct banks.
//   pass : V+ V- D1+ D1- D2+ D2- H+ H-.  Lanes own consecutive disparity
//          pairs; d-1/d+1 neighbours by byte permutes plus one shuffle each
//          way; u16x2 min/max; min over d by redux.sync.  The aggregation
//          volume S ([y][x][64*PPL] u16 in HBM) is stored by the first pass,
//          read-modify-written by the middle ones and read by the last (H-),
//          which finishes S in registers and reduces it to disparities (WTA,
//          right-view disparity, left-right check) without storing it.
//   Vertical and diagonal passes run row-synchronous blocks: G warps own G
//   adjacent path lines and advance one image row per step; per row one
//   thread issues TMA bulk copies (cp.async.bulk) of the S chunk, the left
//   plane entries and the shared right-plane segment into a ring of shared
//   memory slots completed by mbarriers.  Horizontal passes give each warp a
//   row fed by a producer warp (an S ring and a ring of right-plane chunks,
//   TMA bulk copies); the right-plane entries a warp's lanes need slide
//   through a register window, one shuffle and one edge-lane load per step.
//   Every mbarrier wait is bounded; a wait that runs out
//   records TDV_ERR_TIMEOUT, waits (bounded) for its copies in flight and
//   returns.
//
// Reference semantics.  tdvision/semiglobalcpu.cpp:56-126 differs from the
// STANDARD recurrence in the minimum m' it subtracts, taken over d < D-1
// only (:95-97), and its sequential walk loop (:210-222) over the stale path
// table (tdvision/semiglobal.cu:163-166,197-205) with start-assign (:79-83)
// changes only how many times each direction's path cost counts in a cell:
// S(p) = sum_k n_k(p) L_k(p).  The kernels walk every line once and weigh
// each cell's contribution by a class from build_fused_weights: 1 adds L, 0
// adds nothing, 2 adds L and leaves the line's L in a side row, from which
// the last pass adds (n-1) L more in 32-bit arithmetic.  Without the D-1
// term m' can exceed a path cost, so L can go below zero (down to
// -(255 + max(P1, P2-P1))): every direction adds its values with an offset
// OFF = 2*(255 + max(P1, P2-P1)) half-units, folded into the recurrence's
// subtraction of m', and a class-0 cell adds OFF alone, so every cell's S
// carries 8*OFF and cells stay comparable in the left-right check.  The
// sentinel becomes BIG = OFF + 511 + 2*P2h.  The last pass's keys are signed
// (a corrected sum can be negative).  The reference's GPU recurrence
// (tdvision/semiglobal.cu:283-466, without its race) accumulates at path
// starts and differs from STANDARD only in its second step, which sees the
// first costs plus P1 with the minimum of the first costs (GSTART).
//
// This header holds the device code of those passes as __device__ bodies that
// take their block index and shared-memory base explicitly, so that the
// per-frame kernels (kernels_fused.cu, one launch per pass) and the
// persistent batch kernel (kernels_batch.cu, one launch per batch of pairs)
// run the same code.
#pragma once

#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <type_traits>

#include "tdv_internal.hpp"

namespace tdv {

namespace {

constexpr int kMaxG = 24;       // consumer warps per block, vertical/diagonal passes
constexpr int kRowSlots = 8;    // rows in flight, vertical/diagonal passes (power of 2)
constexpr int kVdRowsPerSlot = 2;  // rows per ring slot (one wait and one release per slot)
constexpr int kHSlots = 8;      // S ring depth (steps), horizontal passes
constexpr int kChunk = 64;      // right-plane entries per horizontal refill
constexpr int kChunkSlots = 8;  // resident chunks per horizontal warp
constexpr int kChunk2 = 32;     // right-plane entries per refill, split-D horizontal passes
constexpr int kMaxRowsH2 = 8;   // rows (2 warps each) per block, split-D horizontal passes
constexpr int kLookC = 2;       // chunks fetched ahead of need
constexpr uint64_t kWaitNs = 1000000000ull;   // 1 s: a wait this long means a lost copy
constexpr uint64_t kDrainNs = 10000000ull;    // 10 ms per wait while retiring after an error
constexpr int kGroupBytes = 9 * 16;
constexpr int kChunkBytes = (kChunk / 8) * kGroupBytes;
constexpr uint32_t FULL = 0xFFFFFFFFu;

struct __align__(16) Plane {
    uint32_t i, mn, mx, pad;
};

__host__ __device__ inline int padded_len(int W) { return 9 * ((W + 7) / 8); }
__host__ __device__ inline int align128(int v) { return (v + 127) & ~127; }
__device__ __forceinline__ int ppos(int e) { return e + (e >> 3); }
// Left-plane entry load: through the read-only path when the planes were
// written by an earlier launch, through L2 when a producer in the same
// (persistent) launch may have written them.
__device__ __forceinline__ uint4 ld_plane(const void* p, bool nc) {
    return nc ? __ldg((const uint4*)p) : __ldcg((const uint4*)p);
}

// ------------------------------------------------- tile sizes (host + device)
// Disparity pairs per lane: 64 disparities per warp-row of 32 lanes per pair.
__host__ __device__ inline int ppl_for(int D) { return D <= 64 ? 1 : (D <= 128 ? 2 : 4); }
constexpr int kSmemBudget = 220 * 1024;  // dynamic shared memory per block

// vertical/diagonal pass, G lines: barriers + kRowSlots ring slots of
// (S chunk, left entries, shared right segment) + the diagonal offset tables
// (8 phases x 4 words per warp)
__host__ __device__ inline int vd_smem_bytes(int G, int ppl) {
    const int NRG = (G + 64 * ppl) / 8 + 2;
    return 2 * kRowSlots * 8 + kRowSlots * align128(G * 128 * ppl + G * 16 + NRG * kGroupBytes) + G * 128;
}
// horizontal pass, two warps per row: per warp, then per row (exchange + L-R rows)
__host__ __device__ inline int h2_warp_bytes(int ph) {
    return align128(128 + kHSlots * 128 * ph + kChunkSlots * (kChunk2 / 8) * kGroupBytes);
}
__host__ __device__ inline int h2_row_bytes(bool lr, int W) { return align128(128 + (lr ? 2 * W * 2 : 0)); }

// Rows spanned by the path lines [kf, kf+Gb) of a vertical (s = 0) or
// diagonal (s = +-1) pass, x = kp + s*y (the bounds vd_body walks).
__host__ __device__ inline int group_rows(int W, int H, int s, int kf, int Gb) {
    if (s == 0) return H;
    int ylo, yhi;
    if (s > 0) {
        ylo = max(0, -(kf + Gb - 1));
        yhi = min(H - 1, W - 1 - kf);
    } else {
        ylo = max(0, kf - W + 1);
        yhi = min(H - 1, kf + Gb - 1);
    }
    return max(0, yhi - ylo + 1);
}

// ---------------------------------------------------------------- PTX
__device__ __forceinline__ uint32_t vmin2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t vmax2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("max.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
// (hi16(a), lo16(b)) as (lo, hi) of the result
__device__ __forceinline__ uint32_t hi_lo(uint32_t a, uint32_t b) { return __byte_perm(a, b, 0x5432); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(uint32_t bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
// Slot reuse needs no proxy fence: every generic read of a ring slot feeds
// arithmetic that precedes the release of the slot (mbarrier arrive or warp
// sync), so those reads have completed before the refill is issued.
// 1-D TMA bulk copy global -> shared, completion counted on `bar`.
__device__ __forceinline__ void tma_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for phase `parity` of `bar`: false once `limit_ns` of wall
// time have passed without the phase completing.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint64_t limit_ns = kWaitNs) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

// ---------------------------------------------------------------- planes
__device__ __forceinline__ int u8_at(const ImgArg& im, int x, int y) {
    x = min(max(x, 0), im.W - 1);
    y = min(max(y, 0), im.H - 1);
    return ((const uint8_t*)im.ptr)[(size_t)y * im.pitch + x];
}

// Per pixel, in half-units: 2I, min(2I, I+I(x-1), I+I(x+1)), max(...) with
// clamp-to-edge taps (tdvision/birchfieldcost.cu:22-32).
__device__ __forceinline__ void bt_triple(const ImgArg& im, int x, int y, uint32_t& i2,
                                          uint32_t& mn, uint32_t& mx) {
    const int v = u8_at(im, x, y);
    const int a = v + u8_at(im, x - 1, y);
    const int b = v + u8_at(im, x + 1, y);
    i2 = 2 * v;
    mn = min(2 * v, min(a, b));
    mx = max(2 * v, max(a, b));
}

__device__ __forceinline__ void prep_pixel(const ImgArg& L, const ImgArg& R, Plane* LP, Plane* RPp, int W,
                                           int Wp, int x, int y) {
    uint32_t i2, mn, mx;
    bt_triple(L, x, y, i2, mn, mx);
    Plane lp;
    lp.i = i2 * 0x10001u;
    lp.mn = mn * 0x10001u;
    lp.mx = mx * 0x10001u;
    lp.pad = 0;
    LP[(size_t)y * W + x] = lp;
    uint32_t j2, jn, jx, k2, kn, kx;
    bt_triple(R, x, y, j2, jn, jx);
    bt_triple(R, max(x - 1, 0), y, k2, kn, kx);
    Plane rp;
    rp.i = j2 | (k2 << 16);
    rp.mn = jn | (kn << 16);
    rp.mx = jx | (kx << 16);
    rp.pad = 0;
    RPp[(size_t)y * Wp + x + (x >> 3)] = rp;
}

struct FK {
    const Plane* LP;
    const Plane* RPp;  // padded rows of Wp entries
    uint32_t* S;       // aggregation volume, u16 pairs
    const uint32_t* S2;  // second volume summed by a two-volume last pass (else null)
    int W, H, D, Dp2, Wp;
    uint32_t P1P1, P2P2, BIGBIG;
    uint16_t* disp;
    float* disp_norm;
    uint16_t* disp_right;
    int lr_thr;
    int* err;
    // reference semantics (all zero / null for the STANDARD recurrence over the FULL table)
    uint32_t OFFOFF;          // per-direction offset, half-units in both halves
    const uint8_t* lw;        // this pass's line classes (+4: border cells differ), null: all 1
    const uint8_t* bw;        // this pass's border-cell classes, null: as the line
    uint32_t* side;           // this pass's repeated-line rows (Dp2 words per row)
    const int* corner;        // last pass: per row two (x or -1, (n-1) << 1 | slot) entries
    const uint32_t* side_all; // last pass: the side rows of both slots, slot * H * Dp2
    uint32_t GSTART;          // reference GPU recurrence: P1 (both halves) added to a line's
                              // first path costs before its second step (else 0)
};

// ---------------------------------------------------------------- compute
template <int PPL>
struct Vec;
template <>
struct Vec<1> {
    static __device__ __forceinline__ void st(uint32_t* p, const uint32_t* v) { __stcs(p, v[0]); }
    static __device__ __forceinline__ void lds(const uint32_t* p, uint32_t* v) { v[0] = p[0]; }
};
template <>
struct Vec<2> {
    static __device__ __forceinline__ void st(uint32_t* p, const uint32_t* v) {
        __stcs((uint2*)p, make_uint2(v[0], v[1]));
    }
    static __device__ __forceinline__ void lds(const uint32_t* p, uint32_t* v) {
        const uint2 t = *(const uint2*)p;
        v[0] = t.x;
        v[1] = t.y;
    }
};
template <>
struct Vec<4> {
    static __device__ __forceinline__ void st(uint32_t* p, const uint32_t* v) {
        __stcs((uint4*)p, make_uint4(v[0], v[1], v[2], v[3]));
    }
    static __device__ __forceinline__ void lds(const uint32_t* p, uint32_t* v) {
        const uint4 t = *(const uint4*)p;
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    }
};

// Compile-time loop: f(integral_constant<int, I>) for I in [I0, N).
template <int I, int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
    if constexpr (I < N) {
        f(std::integral_constant<int, I>{});
        static_for<I + 1, N>(f);
    }
}

// BT of one disparity pair from a left entry and a right entry.
__device__ __forceinline__ uint32_t bt_pair(const uint4& lp, const uint4& rp) {
    // .x = I, .y = half-sample min, .z = half-sample max
    const uint32_t A = vmax2(lp.x, rp.y) - vmin2(lp.x, rp.z);
    const uint32_t B = vmax2(rp.x, lp.y) - vmin2(rp.x, lp.z);
    return vmin2(A, B);
}

// Invalid halves (d > x or d >= D) carry BIG.
__device__ __forceinline__ uint32_t mask_pair(uint32_t v, int d, int lim, uint32_t BIGBIG) {
    if (d + 1 >= lim) v = (d < lim) ? ((v & 0xFFFFu) | (BIGBIG & 0xFFFF0000u)) : BIGBIG;
    return v;
}

// Minimum over the warp's disparities.  EXCL leaves out the half that holds
// d = D-1 (the reference CPU recurrence): EXCL 1 when D fills the warp's span
// (D-1 is the high half of lane 31's last pair: one predicated OR, no
// register), EXCL 2 otherwise (exm[q]: 0xFFFF in that half of that lane's
// pair q, else 0).
template <int PPL, int EXCL>
__device__ __forceinline__ uint32_t warp_min_pairs(const uint32_t* L, const uint32_t* exm, bool last_lane) {
    auto val = [&](int q) {
        uint32_t v = L[q];
        if (EXCL == 1 && q == PPL - 1 && last_lane) v |= 0xFFFF0000u;
        if (EXCL == 2) v |= exm[q];
        return v;
    };
    // the pair that may hold D-1 first: the recurrence produces it first, so
    // its mask overlaps the other pairs' work
    uint32_t t = val(PPL - 1);
    #pragma unroll
    for (int q = 0; q < PPL - 1; q++) t = vmin2(t, val(q));
    t = min(t & 0xFFFFu, t >> 16);
    return __reduce_min_sync(FULL, t);
}
// The exclusion mask of lane `lane` (pairs (base_d + 2q, base_d + 2q + 1)).
template <int PPL>
__device__ __forceinline__ void excl_mask(int base_d, int D, uint32_t* exm) {
    #pragma unroll
    for (int q = 0; q < PPL; q++) {
        const int d = base_d + 2 * q;
        exm[q] = d == D - 1 ? 0x0000FFFFu : (d + 1 == D - 1 ? 0xFFFF0000u : 0u);
    }
}

// One step of the min-plus recurrence for this lane's pairs; OFFSET: the
// per-direction offset of the reference CPU recurrence may be nonzero.
template <int PPL, bool OFFSET>
__device__ __forceinline__ void recur(const uint32_t* L, uint32_t m, const uint32_t* c, uint32_t* Ln,
                                      int lane, const FK& k) {
    // L = C + tv - m' + OFF per half: the 32-bit sum is exact modulo 2^32 and
    // each half's result lies in [0, 65535], so no half borrows from the other
    const uint32_t MM = m * 0x10001u;
    const uint32_t MP2 = MM + k.P2P2;
    const uint32_t MMO = OFFSET ? MM - k.OFFOFF : MM;
    uint32_t up = __shfl_up_sync(FULL, L[PPL - 1], 1);
    uint32_t dn = __shfl_down_sync(FULL, L[0], 1);
    if (lane == 0) up = k.BIGBIG;
    if (lane == 31) dn = k.BIGBIG;
    #pragma unroll
    for (int qq = 0; qq < PPL; qq++) {
        const int q = PPL - 1 - qq;  // the last pair first (see warp_min_pairs)
        const uint32_t lm = hi_lo(q > 0 ? L[q - 1] : up, L[q]);
        const uint32_t lp = hi_lo(L[q], q < PPL - 1 ? L[q + 1] : dn);
        uint32_t tv = vmin2(lm, lp) + k.P1P1;
        tv = vmin2(vmin2(tv, L[q]), MP2);
        Ln[q] = tv + c[q] - MMO;
    }
}

// ---------------------------------------------- vertical / diagonal passes
// A path line is x = kp + s*y (s = dx*dy); the block owns lines
// j0 .. j0+G-1 (kp = kmin + j) and walks rows in the pass direction dy.
// Warps 0..G-1 consume one row per step; warp G is the producer: its lane 0
// issues the TMA copies of row i into ring slot i % kRowSlots once every
// consumer warp has released the slot's previous row (full/empty mbarrier
// pairs), so no block-wide barrier is taken per row.  DIAG = false (s = 0):
// a line is one column, so each lane's right-plane offsets are the same on
// every row and are computed once; the recurrence starts from L = 0, m = 0
// (first step L = C, as in the horizontal passes).
// VAR 0: the STANDARD recurrence over the full table (no weight, offset or
// first-step code is compiled in); 1: weights / reference recurrences, 2: as
// 1 with the excluded minimum of D-1 at lane 31 (D fills the span), 3: as 1
// with the excluded minimum anywhere.
template <int PPL, int MODE, bool DIAG, int VAR = 0>
__device__ __forceinline__ void vd_body(const FK& k, int s, int dy, int kmin, int nlines, int G, int blk,
                                        unsigned char* smem) {
    constexpr bool WTD = VAR != 0;
    constexpr int EXCL = VAR == 2 ? 1 : (VAR == 3 ? 2 : 0);
    constexpr int SB = 128 * PPL;
    constexpr int DSPAN = 64 * PPL;
    constexpr int U = kVdRowsPerSlot;
    constexpr int NS = kRowSlots / U;  // ring slots (power of 2)
    const int NRG = (G + DSPAN) / 8 + 2;
    const int offL = G * SB, offR = offL + G * 16;
    const int rowBytes = align128(offR + NRG * kGroupBytes);
    const int slotBytes = U * rowBytes;
    uint64_t* full = (uint64_t*)smem;
    uint64_t* empty = full + NS;
    unsigned char* slots = smem + 2 * kRowSlots * 8;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j0 = blk * G;
    const int Gb = min(G, nlines - j0);
    const int kf = kmin + j0;
    int ylo, yhi;
    if (s == 0) {
        ylo = 0;
        yhi = k.H - 1;
    } else if (s > 0) {
        ylo = max(0, -(kf + Gb - 1));
        yhi = min(k.H - 1, k.W - 1 - kf);
    } else {
        ylo = max(0, kf - k.W + 1);
        yhi = min(k.H - 1, kf + Gb - 1);
    }
    const int nrows = yhi - ylo + 1;
    if (nrows <= 0) return;  // uniform for the block
    const int y0 = dy > 0 ? ylo : yhi;
    const int nslots = (nrows + U - 1) / U;

    if (threadIdx.x == 0) {
        for (int b = 0; b < NS; b++) {
            mbar_init(smem_u32(&full[b]), 1);
            mbar_init(smem_u32(&empty[b]), Gb);  // warps without a line take no part
        }
        fence_mbar_init();
    }
    __syncthreads();

    if (warp == G) {
        // ---- producer: slot j holds rows U*j .. U*j+U-1 ----
        if (lane == 0) {
            int j = 0;
            bool ok = true;
            for (; j < nslots; j++) {
                const int b = j & (NS - 1);
                if (j >= NS && !mbar_wait(smem_u32(&empty[b]), (uint32_t)((j / NS) - 1) & 1u)) {
                    ok = false;
                    break;
                }
                const uint32_t bar = smem_u32(&full[b]);
                // the right-plane segment of a row starts (virtually) at group
                // g0v = floor((xf - DSPAN + 2) / 8), which may be negative:
                // groups left of the image are not copied (their cells are masked)
                uint32_t total = 0;
                for (int r = 0; r < U && U * j + r < nrows; r++) {
                    const int y = y0 + dy * (U * j + r);
                    const int xf = kf + s * y;
                    const int xlo = max(xf, 0), xhi = min(xf + Gb, k.W);
                    const int g0 = max(0, (xf - DSPAN + 2) >> 3), g1 = (xhi - 1) >> 3;
                    total += (uint32_t)(xhi - xlo) * ((MODE != 0 ? SB : 0) + 16) + (uint32_t)(g1 - g0 + 1) * kGroupBytes;
                }
                mbar_expect_tx(bar, total);
                for (int r = 0; r < U && U * j + r < nrows; r++) {
                    const int y = y0 + dy * (U * j + r);
                    const int xf = kf + s * y;
                    const int xlo = max(xf, 0), xhi = min(xf + Gb, k.W);
                    const int npx = xhi - xlo;
                    const int g0v = (xf - DSPAN + 2) >> 3;  // arithmetic shift: floor division
                    const int g0 = max(0, g0v), g1 = (xhi - 1) >> 3;
                    unsigned char* base = slots + b * slotBytes + r * rowBytes;
                    if (MODE != 0)
                        tma_load(smem_u32(base + (xlo - xf) * SB), k.S + ((size_t)y * k.W + xlo) * k.Dp2,
                                 (uint32_t)npx * SB, bar);
                    tma_load(smem_u32(base + offL + (xlo - xf) * 16), k.LP + (size_t)y * k.W + xlo,
                             (uint32_t)npx * 16, bar);
                    tma_load(smem_u32(base + offR + (g0 - g0v) * kGroupBytes), k.RPp + (size_t)y * k.Wp + 9 * g0,
                             (uint32_t)(g1 - g0 + 1) * kGroupBytes, bar);
                }
            }
            if (!ok) atomicExch(k.err, (int)TDV_ERR_TIMEOUT);
            // the block must not retire with copies in flight
            for (int r = max(0, j - NS); r < j; r++)
                mbar_wait(smem_u32(&full[r & (NS - 1)]), (uint32_t)(r / NS) & 1u, ok ? kWaitNs : kDrainNs);
        }
    } else if (warp < Gb) {
        // ---- consumers: warp w walks line kf + w ----
        const int base_d = lane * 2 * PPL;
        const bool dmask = k.D < DSPAN;  // some lanes hold disparities >= D
        const unsigned char* lp_slot = slots + offL + warp * 16;
        const unsigned char* sv_slot = slots + warp * SB + lane * PPL * 4;
        uint32_t L[PPL], m = 0, exm[PPL];
#pragma unroll
        for (int q = 0; q < PPL; q++) L[q] = 0;
        if (EXCL == 2) excl_mask<PPL>(base_d, k.D, exm);
        const bool last_lane = lane == 31;
        bool started = false;  // the line's first cell has been walked
        // weight class of the line (reference table / recurrence): 0 counts
        // nowhere, 1 counts once, 2 the repeated line (leaves side rows); lbw:
        // some border cells of the line have classes of their own
        const int lwv = (WTD && k.lw) ? (int)k.lw[j0 + warp] : 1;
        const int lcls = WTD ? (lwv & 3) : 1;
        const bool lbw = WTD && k.bw && (lwv & 4);
        // vertical (s = 0): column x = kp on every row, offsets computed once
        const int xs = kf + warp;
        const int lim_s = min(xs + 1, k.D);
        // right-plane entry e of a row sits at ppos(e - 8*g0v) in the segment
        // (g0v its virtual first group, a multiple of 8 entries below e): for
        // the line x = xf + warp that is ppos(cq + phase), with the per-lane
        // constant cq = DSPAN - 2 + warp - base_d - 2q and the per-row phase
        // (xf - DSPAN + 2) & 7; vertical lines have one phase for every row
        int cq[PPL], rpos[PPL];
#pragma unroll
        for (int q = 0; q < PPL; q++) {
            cq[q] = DSPAN - 2 + warp - base_d - 2 * q;
            rpos[q] = ppos(cq[q] + ((kf - DSPAN + 2) & 7)) * 16;
        }
        // With four pairs per lane (base_d = 8 * lane, a whole group of
        // entries per lane) the offset splits as ppos(phase + C_q) * 16 -
        // 144 * lane, C_q = DSPAN - 2 + warp - 2q: the first term depends on
        // the warp, the pair and the row's phase only, so each warp keeps it
        // in a table of 8 phases x 4 pairs and a diagonal row reads one entry.
        const uint32_t* tbl = (const uint32_t*)(slots + kRowSlots * rowBytes) + warp * 32;
        if constexpr (DIAG && PPL == 4) {
            if (lane < 8) {
                uint32_t* t = (uint32_t*)(slots + kRowSlots * rowBytes) + warp * 32 + lane * 4;
#pragma unroll
                for (int q = 0; q < 4; q++) t[q] = (uint32_t)ppos(lane + DSPAN - 2 + warp - 2 * q) * 16u;
            }
            __syncwarp();
        }
        const int rlane = offR - 144 * lane;
        // the line's S vector on row y0, and the step to the next row (x moves by s*dy)
        uint32_t* sg = k.S + ((long long)y0 * k.W + xs + s * y0) * k.Dp2 + lane * PPL;
        const long long sstep = (long long)dy * (k.W + s) * k.Dp2;

        // CHECK: the row may lie outside the line's span (diagonal) or hold
        // cells with d > x or d >= D; without it the row is known clean
        // the repeated line's side row of the current walk row
        uint32_t* sidep = (WTD && DIAG && lcls == 2) ? k.side + (size_t)y0 * k.Dp2 + lane * PPL : nullptr;
        const long long sidestep = (long long)dy * k.Dp2;
        // CHECK: masking and the diagonal span; SPEC (implies CHECK): the
        // weight classes, the side rows and the first cell of a line
        auto row = [&](auto chk, auto spc, int i, int boff) {
            constexpr bool SPEC = decltype(spc)::value;
            constexpr bool CHECK = decltype(chk)::value || SPEC;
            uint32_t c[PPL], Ln[PPL];
            const int yc = CHECK ? y0 + dy * i : 0;
            const int xc = CHECK ? xs + s * yc : 0;
            if (DIAG && CHECK && (xc < 0 || xc >= k.W)) {  // uniform: one line per warp
                sg += sstep;
                if constexpr (WTD && DIAG) sidep += sidestep;
                return;
            }
            if (SPEC && lcls == 0) {
                // no walk of this direction: every cell adds the offset alone
                uint32_t sv[PPL];
                if (MODE == 0) {
#pragma unroll
                    for (int q = 0; q < PPL; q++) sv[q] = k.OFFOFF;
                } else {
                    Vec<PPL>::lds((const uint32_t*)(sv_slot + boff), sv);
#pragma unroll
                    for (int q = 0; q < PPL; q++) sv[q] += k.OFFOFF;
                }
                Vec<PPL>::st(sg, sv);
                sg += sstep;
                if constexpr (WTD && DIAG) sidep += sidestep;
                return;
            }
            if (!DIAG) {
                const uint4 lp = *(const uint4*)(lp_slot + boff);
#pragma unroll
                for (int q = 0; q < PPL; q++) c[q] = bt_pair(lp, *(const uint4*)(slots + offR + boff + rpos[q]));
                if (CHECK) {
#pragma unroll
                    for (int q = 0; q < PPL; q++) c[q] = mask_pair(c[q], base_d + 2 * q, lim_s, k.BIGBIG);
                }
            } else {
                const int y = y0 + dy * i;
                const int x = xs + s * y;
                const uint4 lp = *(const uint4*)(lp_slot + boff);
                const int phase = (kf + s * y - DSPAN + 2) & 7;
                if constexpr (PPL == 4) {
                    const uint4 A = *(const uint4*)(tbl + phase * 4);
                    const unsigned char* rb = slots + (boff + rlane);
                    c[0] = bt_pair(lp, *(const uint4*)(rb + A.x));
                    c[1] = bt_pair(lp, *(const uint4*)(rb + A.y));
                    c[2] = bt_pair(lp, *(const uint4*)(rb + A.z));
                    c[3] = bt_pair(lp, *(const uint4*)(rb + A.w));
                } else {
                    const unsigned char* rseg = slots + boff + offR;
#pragma unroll
                    for (int q = 0; q < PPL; q++)
                        c[q] = bt_pair(lp, *(const uint4*)(rseg + ppos(cq[q] + phase) * 16));
                }
                if (CHECK && (x < DSPAN || dmask)) {
                    const int lim = min(x + 1, k.D);
#pragma unroll
                    for (int q = 0; q < PPL; q++) c[q] = mask_pair(c[q], base_d + 2 * q, lim, k.BIGBIG);
                }
            }
            recur<PPL, WTD>(L, m, c, Ln, lane, k);  // from L = 0, m = 0 the first step gives L = C (+ OFF)
            uint32_t add[PPL];
#pragma unroll
            for (int q = 0; q < PPL; q++) add[q] = Ln[q];
            if (SPEC) {
                // a border cell whose sum a later walk restarts counts the offset alone
                if (lbw && (yc == 0 || yc == k.H - 1 || xc == 0 || xc == k.W - 1) &&
                    k.bw[border_index(k.W, k.H, xc, yc)] == 0) {
#pragma unroll
                    for (int q = 0; q < PPL; q++) add[q] = k.OFFOFF;
                }
            }
            // the repeated line leaves its path costs in the side rows (one
            // line per warp: a predicated store in every row variant)
            if constexpr (WTD && DIAG) {
                if (lcls == 2) Vec<PPL>::st(sidep, Ln);
            }
            if (MODE == 0) {
                Vec<PPL>::st(sg, add);
            } else {
                uint32_t sv[PPL];
                Vec<PPL>::lds((const uint32_t*)(sv_slot + boff), sv);
#pragma unroll
                for (int q = 0; q < PPL; q++) sv[q] += add[q];
                Vec<PPL>::st(sg, sv);
            }
            sg += sstep;
            if constexpr (WTD && DIAG) sidep += sidestep;
#pragma unroll
            for (int q = 0; q < PPL; q++) L[q] = Ln[q];
            m = warp_min_pairs<PPL, EXCL>(L, exm, last_lane);
            if (SPEC && k.GSTART && !started) {
                // reference GPU recurrence: the second step sees C + P1 with
                // the minimum of C (tdvision/semiglobal.cu:353-358)
#pragma unroll
                for (int q = 0; q < PPL; q++) L[q] += k.GSTART;
            }
            if (SPEC) started = true;
        };

        // a vertical line needs masking on every row or on none; lines that
        // count nowhere, and border columns with classes of their own, take
        // the special rows throughout
        const bool vcheck = !DIAG && (xs < DSPAN || dmask);
        const bool vspec = WTD && (lcls == 0 || (lbw && !DIAG && (xs == 0 || xs == k.W - 1)));
        // the slots that hold the line's first and last cells in walk order:
        // a line's border cells are its two end cells (besides whole border
        // columns, above), and the reference GPU recurrence treats the first
        // cell's successor apart
        int jsa = -1, jsb = -1;
        if (WTD && (lbw || k.GSTART)) {
            int yf = 0, yl = k.H - 1;
            if (DIAG) {
                const int kp = kf + warp;
                yf = s > 0 ? max(0, -kp) : max(0, kp - (k.W - 1));
                yl = s > 0 ? min(k.H - 1, k.W - 1 - kp) : min(k.H - 1, kp);
            }
            if (dy < 0) {
                const int t = yf;
                yf = yl;
                yl = t;
            }
            jsa = (yf - y0) * dy / U;
            jsb = lbw ? (yl - y0) * dy / U : jsa;
        }
        for (int j = 0; j < nslots; j++) {
            const int b = j & (NS - 1);
            if (!__all_sync(FULL, mbar_wait(smem_u32(&full[b]), (uint32_t)(j / NS) & 1u))) {
                if (lane == 0) atomicExch(k.err, (int)TDV_ERR_TIMEOUT);
                break;
            }
            const int boff = b * slotBytes;
            const bool full_slot = U * j + U <= nrows;
            bool check = vcheck || !full_slot;
            const bool spec = WTD && (vspec || j == jsa || j == jsb);
            if (DIAG) {
                // x = xs + s*y is monotone over the slot's rows: check its ends
                const int xa = xs + s * (y0 + dy * (U * j)), xb = xa + s * dy * (U - 1);
                check = check || min(xa, xb) < DSPAN || max(xa, xb) >= k.W || dmask;
            }
            if (spec) {
                if constexpr (WTD) {
#pragma unroll
                    for (int r = 0; r < U; r++)
                        if (U * j + r < nrows) row(std::true_type{}, std::true_type{}, U * j + r, boff + r * rowBytes);
                }
            } else if (check) {
#pragma unroll
                for (int r = 0; r < U; r++)
                    if (U * j + r < nrows) row(std::true_type{}, std::false_type{}, U * j + r, boff + r * rowBytes);
            } else {
#pragma unroll
                for (int r = 0; r < U; r++) row(std::false_type{}, std::false_type{}, U * j + r, boff + r * rowBytes);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&empty[b]));
        }
    }
    // every role is done with the ring: retire its barriers so that the
    // shared memory can be reused by the next work item (whose TMA writes
    // must follow this item's generic reads)
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0)
        for (int b = 0; b < 2 * NS; b++) mbar_inval(smem_u32(&full[b]));
}

// ------------------------------------- horizontal passes, producer-fed
// R consumer warps (one image row each, walking x in direction dx) and one
// producer warp whose lane r keeps row r's rings full, so the consumers carry
// no copy bookkeeping.  Per row:
//   * an S ring of hp_slots(TWO) slots, each holding hp_px(TWO) consecutive pixels of
//     the row: their S vectors and their left-plane entries (two TMA bulk
//     copies per slot); a consumer waits once per slot and releases the
//     slot (mbarrier arrive) when it has read it;
//   * a right-plane chunk ring of kHpChunkSlots chunks of kChunk entries,
//     chunk c in slot c & 3, read only by the lane that loads the entry
//     entering the warp's register window; the consumer releases a chunk
//     once the loads have passed it, the producer refills the slot with the
//     chunk 4 places further in walk order.
// The producer lanes never block: each polls its own row's empty barriers and
// issues what has become free; the warp pauses 256 ns after every round and
// gives up (TDV_ERR_TIMEOUT) after kWaitNs without progress.
// The recurrence starts from L = 0, m = 0, which makes the first step L = C
// without a branch (min(0, 0 + P1, 0 + P2) = 0).
// TWO: the pass joins two volumes filled by concurrent pass chains, k.S and
// k.S2 (read-only): a slot also holds the S2 vectors, and the pass stores
// S + S2 + L into k.S.
constexpr int kHpChunkSlots = 4;  // right-plane chunks per row (power of 2)
// Pixels per S slot and S slots per row.  A slot of 8 pixels matches the
// eight-step unroll: one slot wait per iteration, so the eight steps are one
// straight-line stretch the compiler schedules across (a wait is an asm
// barrier to it), and 4 KB copies per volume.  The two-volume join holds two
// such slots per row, the other passes three.
__host__ __device__ constexpr int hp_px(bool) { return 8; }
__host__ __device__ constexpr int hp_slots(bool two) { return two ? 2 : 3; }
__host__ __device__ constexpr int hp_bars(bool two) { return 2 * hp_slots(two) + 2 * kHpChunkSlots; }

// slot: [S vectors of hp_px(two) pixels][S2 vectors (TWO)][left-plane entries],
// padded to 128 bytes so every slot's vectors start on a 128-byte line
__host__ __device__ inline int hp_slot_bytes(int ppl, bool two) {
    return align128(hp_px(two) * (128 * ppl * (two ? 2 : 1) + 16));
}
__host__ __device__ inline int hp_warp_bytes(int ppl, bool lr, int W, bool two) {
    return align128(hp_slots(two) * hp_slot_bytes(ppl, two) + kHpChunkSlots * kChunkBytes + (lr ? 2 * W * 2 : 0));
}
__host__ __device__ inline int hp_smem_bytes(int R, int ppl, bool lr, int W, bool two) {
    return align128(R * hp_bars(two) * 8) + R * hp_warp_bytes(ppl, lr, W, two);
}

// The last pass's keys of a cell that counts a repeated line more than once:
// the cell's packed 16-bit sums plus (n-1) L from the side row(s) of its row,
// as signed 32-bit (S << 8 | d) clamped at 2^23 - 1 so that invalid cells stay
// above every valid one.  Out of line (two cells of a row take it, and the
// horizontal step it would sit in is unrolled many times over); sums and keys
// travel by value so that the callers' arrays stay in registers.
template <int PPL>
struct PairRow {
    uint32_t v[PPL];
};
template <int PPL>
struct KeyRow {
    int v[2 * PPL];
};
template <int PPL>
__device__ __noinline__ KeyRow<PPL> corner_keys(const int* corner, const uint32_t* side_all, int H, int Dp2, int off,
                                                int y, int x, uint32_t cxs, int lane, int base_d, PairRow<PPL> sv) {
    KeyRow<PPL> r;
#pragma unroll
    for (int q = 0; q < PPL; q++) {
        r.v[2 * q] = (int)(sv.v[q] & 0xFFFFu);
        r.v[2 * q + 1] = (int)(sv.v[q] >> 16);
    }
#pragma unroll
    for (int e = 0; e < 2; e++) {
        if (x != (int)((cxs >> (16 * e)) & 0xFFFFu)) continue;
        const int cc = corner[4 * y + 2 * e + 1];
        const uint32_t* sd = side_all + ((size_t)(cc & 1) * H + y) * Dp2 + lane * PPL;
        const int w = cc >> 1;
#pragma unroll
        for (int q = 0; q < PPL; q++) {
            const uint32_t u = __ldcg(sd + q);
            r.v[2 * q] += w * ((int)(u & 0xFFFFu) - off);
            r.v[2 * q + 1] += w * ((int)(u >> 16) - off);
        }
    }
#pragma unroll
    for (int j = 0; j < 2 * PPL; j++) r.v[j] = min(r.v[j], (1 << 23) - 1) * 256 + base_d + j;
    return r;
}

template <int PPL, int MODE, bool TWO, int VAR = 0>
__device__ __forceinline__ void hp_body(const FK& k, int dx, int R, int blk, unsigned char* smem) {
    constexpr bool WTD = VAR != 0;  // VAR as for vd_body
    constexpr int EXCL = VAR == 2 ? 1 : (VAR == 3 ? 2 : 0);
    constexpr int SB = 128 * PPL;
    constexpr int NSL = hp_slots(TWO);   // S slots per row
    constexpr int kHpU = hp_px(TWO);     // pixels per S slot
    constexpr int CS = kHpChunkSlots;    // right-plane chunks per row
    constexpr int BARS = hp_bars(TWO);
    constexpr int DSPAN = 64 * PPL;
    constexpr int NJ = 2 * PPL;
    constexpr int SLOT = (kHpU * ((TWO ? 2 : 1) * SB + 16) + 127) & ~127;
    constexpr int LPOFF = kHpU * (TWO ? 2 : 1) * SB;  // left-plane entries in a slot
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = k.W;
    const bool lr = MODE == 2 && k.lr_thr >= 0;
    const int wb = hp_warp_bytes(PPL, lr, W, TWO);
    uint64_t* bars = (uint64_t*)smem;
    unsigned char* data = smem + align128(R * BARS * 8);
    const int y0 = blk * R;
    const int Rb = min(R, k.H - y0);  // rows of this block
    const int ngroups = (W + kHpU - 1) / kHpU;
    const int nch = (W + kChunk - 1) / kChunk;
    const int c0 = dx > 0 ? 0 : nch - 1;  // first chunk in walk order
    // row r: fullS[NSL] emptyS[NSL] fullC[8] emptyC[8]
    auto fullS = [&](int r, int s) { return smem_u32(&bars[r * BARS + s]); };
    auto emptyS = [&](int r, int s) { return smem_u32(&bars[r * BARS + NSL + s]); };
    auto fullC = [&](int r, int s) { return smem_u32(&bars[r * BARS + 2 * NSL + s]); };
    auto emptyC = [&](int r, int s) { return smem_u32(&bars[r * BARS + 2 * NSL + CS + s]); };
    auto group_lo = [&](int j) { return dx > 0 ? j * kHpU : max(0, W - 1 - j * kHpU - (kHpU - 1)); };
    auto group_hi = [&](int j) { return dx > 0 ? min(W - 1, j * kHpU + kHpU - 1) : W - 1 - j * kHpU; };

    if (threadIdx.x == 0) {
        for (int b = 0; b < R * BARS; b++) mbar_init(smem_u32(&bars[b]), 1);
        fence_mbar_init();
    }
    __syncthreads();

    if (warp == R) {
        // ---- producer: lane r feeds row r ----
        const bool mine = lane < Rb;
        const int y = y0 + lane;
        unsigned char* wbase = data + (size_t)lane * wb;
        int g = 0, kc = 0;
        bool failed = false;
        uint64_t t_last = global_ns();
        for (;;) {
            bool pending = false, did = false;
            if (mine) {
                if (g < ngroups) {
                    pending = true;
                    const int s = g % NSL;
                    if (g < NSL || mbar_try(emptyS(lane, s), (uint32_t)((g / NSL) - 1) & 1u)) {
                        const int xlo = group_lo(g), n = group_hi(g) - xlo + 1;
                        unsigned char* dst = wbase + s * SLOT;
                        const uint32_t bar = fullS(lane, s);
                        mbar_expect_tx(bar, (uint32_t)n * ((TWO ? 2 : 1) * SB + 16));
                        tma_load(smem_u32(dst), k.S + ((size_t)y * W + xlo) * k.Dp2, (uint32_t)n * SB, bar);
                        if (TWO)
                            tma_load(smem_u32(dst + kHpU * SB), k.S2 + ((size_t)y * W + xlo) * k.Dp2,
                                     (uint32_t)n * SB, bar);
                        tma_load(smem_u32(dst + LPOFF), k.LP + (size_t)y * W + xlo, (uint32_t)n * 16, bar);
                        g++;
                        did = true;
                    }
                }
                if (kc < nch) {
                    pending = true;
                    const int c = dx > 0 ? kc : c0 - kc;
                    const int s = c & (CS - 1);
                    if (kc < CS || mbar_try(emptyC(lane, s), (uint32_t)((kc / CS) - 1) & 1u)) {
                        const int ng = min(kChunk / 8, (W + 7) / 8 - c * (kChunk / 8));
                        const uint32_t bar = fullC(lane, s);
                        mbar_expect_tx(bar, (uint32_t)ng * kGroupBytes);
                        tma_load(smem_u32(wbase + NSL * SLOT + s * kChunkBytes),
                                 k.RPp + (size_t)y * k.Wp + 9 * (c * (kChunk / 8)), (uint32_t)ng * kGroupBytes, bar);
                        kc++;
                        did = true;
                    }
                }
            }
            if (!__any_sync(FULL, pending)) break;
            if (__any_sync(FULL, did)) {
                t_last = global_ns();
            } else {
                if (global_ns() - t_last > kWaitNs) {
                    failed = true;
                    break;
                }
            }
            // a pause after every round, work or not: with every row releasing a
            // slot each few hundred ns a busy producer would otherwise poll
            // without rest, taking issue slots from the two consumer warps of
            // its SM sub-partition (a slot's refill still lands well before the
            // slot is needed again)
            __nanosleep(256);
        }
        // the block must not retire with copies in flight
        if (mine) {
            const uint64_t lim = failed ? kDrainNs : kWaitNs;
            for (int j = max(0, g - NSL); j < g; j++)
                mbar_wait(fullS(lane, j % NSL), (uint32_t)(j / NSL) & 1u, lim);
            for (int q = max(0, kc - CS); q < kc; q++) {
                const int c = dx > 0 ? q : c0 - q;
                mbar_wait(fullC(lane, c & (CS - 1)), (uint32_t)(q / CS) & 1u, lim);
            }
        }
        if (failed && lane == 0) atomicExch(k.err, (int)TDV_ERR_TIMEOUT);
    } else if (warp < Rb) {
        // ---- consumer: row y0 + warp ----
        const int r = warp;
        const int y = y0 + r;
        unsigned char* wbase = data + (size_t)r * wb;
        const unsigned char* cring = wbase + NSL * SLOT;
        uint16_t* rowL = (uint16_t*)(cring + CS * kChunkBytes);
        uint16_t* rowR = rowL + W;
        const int base_d = lane * 2 * PPL;
        constexpr int NR = CS * kChunk;  // right-plane entries in the chunk ring
        static_assert(8 % NJ == 0, "the window ring must divide the 8-step unroll");
        uint32_t exm[PPL];
        if (EXCL == 2) excl_mask<PPL>(base_d, k.D, exm);
        const bool last_lane = lane == 31;
        // reference weights: a row counts nowhere (every step adds the offset
        // alone, no recurrence), or once with border cells that may have
        // classes of their own; in the last pass up to two cells of the row
        // count a repeated line more than once
        // the row's state in two registers: flags (1 counts nowhere, 2 border
        // cells with classes of their own, 4 an all-border row of those) and
        // the columns of the repeated cells, 16 bits each (0xFFFF: none;
        // their counts are read again where a group holds one)
        const int rwv = (WTD && k.lw) ? (int)k.lw[y] : 1;
        const bool rbw0 = WTD && k.bw && (rwv & 4);
        const uint32_t rflags = ((rwv & 3) == 0 ? 1u : 0u) | (rbw0 ? 2u : 0u) |
                                (rbw0 && (y == 0 || y == k.H - 1) ? 4u : 0u);
        uint32_t cxs = 0xFFFFFFFFu;
        if (WTD && MODE == 2 && k.corner) {
            const int2 e0 = *(const int2*)(k.corner + 4 * y), e1 = *(const int2*)(k.corner + 4 * y + 2);
            cxs = (e0.x < 0 ? 0xFFFFu : (uint32_t)e0.x) | ((e1.x < 0 ? 0xFFFFu : (uint32_t)e1.x) << 16);
        }

        // One walk of the row in direction DXP (x increasing) with the
        // left-right chain on or off.  Lane l at column x needs the
        // right-plane entries x - base_d - o, o in [0, NJ) (pair q uses
        // o = 2q); they sit in a register window, a ring of NJ entries, and
        // slide one entry per step: the entry a lane no longer needs is the
        // one its neighbour needs next (one shuffle), and the edge lane
        // (lane 0 walking right, lane 31 walking left) loads the entry that
        // enters the warp's window.  Steps run eight at a time (two S slots)
        // so that every ring position is a compile-time index.
        auto consume = [&](auto dxc, auto lrc) -> bool {
            constexpr bool DXP = decltype(dxc)::value;
            constexpr bool LR = decltype(lrc)::value;
            uint32_t L[PPL], m = 0;
            bool started = false;             // the row's first cell has been walked
            uint32_t WI[NJ], WN[NJ], WX[NJ];  // window: I, half-sample min, half-sample max
            int P[NJ];                        // right-view chain (ring, logical j at (T + j) % NJ)
            uint32_t dpair[PPL];              // (d, d+1) of each pair, u16 halves
#pragma unroll
            for (int q = 0; q < PPL; q++) {
                L[q] = 0;
                dpair[q] = (uint32_t)(base_d + 2 * q) | ((uint32_t)(base_d + 2 * q + 1) << 16);
            }
#pragma unroll
            for (int j = 0; j < NJ; j++) {
                WI[j] = WN[j] = WX[j] = 0;
                P[j] = INT_MAX;
            }
            const bool loader = DXP ? lane == 0 : lane == 31;
            uint32_t* sg = k.S + ((size_t)y * W + (DXP ? 0 : W - 1)) * k.Dp2 + lane * PPL;
            const long long sstep = (long long)(DXP ? 1 : -1) * k.Dp2;
            int waited = DXP ? -1 : c0 + 1;  // last chunk waited for
            int rel = c0;                    // next chunk to release
            auto ring_entry = [&](int e) { return *(const uint4*)(cring + ppos(e & (NR - 1)) * 16); };

            // Chunks are waited for in walk order up to the one group j's
            // edge-lane loads reach, and a chunk is released once it has been
            // waited for (its copy has landed) and the edge lane has passed it,
            // so the producer refills slots only after their copies completed.
            // Walking right the edge lane reads entry x; walking left entry
            // x - DSPAN + 1 (clamped at 0), so the chunks a group needs are at
            // most two and a ring of 4 never blocks.
            auto chunks_for = [&](int j) -> bool {
                const int xlo = group_lo(j), xhi = group_hi(j);
                bool good = true;
                if (DXP) {
                    const int keep = xlo >> 6, need = xhi >> 6;
                    auto release = [&]() {
                        if (lane == 0)
                            for (; rel < keep && rel <= waited; rel++) mbar_arrive(emptyC(r, rel & (CS - 1)));
                    };
                    release();
                    while (good && waited < need) {
                        waited++;
                        good = mbar_wait(fullC(r, waited & (CS - 1)), (uint32_t)(waited / CS) & 1u);
                        release();
                    }
                } else {
                    const int keep = max(0, xhi - DSPAN + 1) >> 6, need = max(0, xlo - DSPAN + 1) >> 6;
                    auto release = [&]() {
                        if (lane == 0)
                            for (; rel > keep && rel >= waited; rel--) mbar_arrive(emptyC(r, rel & (CS - 1)));
                    };
                    release();
                    while (good && waited > need) {
                        waited--;
                        good = mbar_wait(fullC(r, waited & (CS - 1)), (uint32_t)((c0 - waited) / CS) & 1u);
                        release();
                    }
                }
                return good;
            };

            // window position T (mod 8); MASK: cells with d > x or d >= D may
            // occur; SPEC (implies MASK): border classes, the repeated-line
            // correction, the row's first cell
            auto step = [&](auto Tc, auto Mc, auto Sc, int x, const unsigned char* slot, int xo) {
                constexpr int T = decltype(Tc)::value;
                constexpr bool SPEC = decltype(Sc)::value;
                constexpr bool MASK = decltype(Mc)::value || SPEC;
                constexpr int N = T % NJ;
                // a row that counts nowhere: no right-plane window, cost or recurrence
                const bool zero = SPEC && (rflags & 1u);
                uint32_t c[PPL], Ln[PPL], sv[PPL];
                if (!zero) {
                    uint32_t vi, vn, vx;
                    if (DXP) {
                        vi = __shfl_up_sync(FULL, WI[N], 1);
                        vn = __shfl_up_sync(FULL, WN[N], 1);
                        vx = __shfl_up_sync(FULL, WX[N], 1);
                    } else {
                        vi = __shfl_down_sync(FULL, WI[N], 1);
                        vn = __shfl_down_sync(FULL, WN[N], 1);
                        vx = __shfl_down_sync(FULL, WX[N], 1);
                    }
                    if (loader) {
                        const uint4 v = ring_entry(DXP ? x : max(x - DSPAN + 1, 0));
                        vi = v.x;
                        vn = v.y;
                        vx = v.z;
                    }
                    WI[N] = vi;
                    WN[N] = vn;
                    WX[N] = vx;
                    const uint4 lp = *(const uint4*)(slot + LPOFF + xo * 16);
#pragma unroll
                    for (int q = 0; q < PPL; q++) {
                        const int w = DXP ? ((T - 2 * q) % NJ + NJ) % NJ : (T + 2 * q + 1) % NJ;
                        c[q] = bt_pair(lp, make_uint4(WI[w], WN[w], WX[w], 0u));
                    }
                    if (MASK) {
                        const int lim = min(x + 1, k.D);
#pragma unroll
                        for (int q = 0; q < PPL; q++) c[q] = mask_pair(c[q], base_d + 2 * q, lim, k.BIGBIG);
                    }
                    recur<PPL, WTD>(L, m, c, Ln, lane, k);
                }
                Vec<PPL>::lds((const uint32_t*)(slot + xo * SB) + lane * PPL, sv);
                if (zero || (SPEC && (rflags & 2u) && ((rflags & 4u) || x == 0 || x == W - 1) &&
                             k.bw[border_index(W, k.H, x, y)] == 0)) {
                    // a border cell a later walk restarts: the offset alone
#pragma unroll
                    for (int q = 0; q < PPL; q++) sv[q] += k.OFFOFF;
                } else if (WTD && !SPEC && (rflags & 1u)) {
                    // a row that counts nowhere walked by the clean or masked
                    // step (cheaper than the special one): its path costs are
                    // computed and dropped, the offset alone is added
#pragma unroll
                    for (int q = 0; q < PPL; q++) sv[q] += k.OFFOFF;
                } else {
#pragma unroll
                    for (int q = 0; q < PPL; q++) sv[q] += Ln[q];
                }
                if (TWO) {
                    uint32_t s2[PPL];
                    Vec<PPL>::lds((const uint32_t*)(slot + kHpU * SB + xo * SB) + lane * PPL, s2);
#pragma unroll
                    for (int q = 0; q < PPL; q++) sv[q] += s2[q];
                }
                if (MODE == 1) {
                    Vec<PPL>::st(sg, sv);
                } else {
                    // WTA key (S << 8 | d): lowest S, then lowest d (tdvision/wtacpu.cpp:26-30);
                    // one byte permute per key from S and the lane's (d, d+1) register.
                    // Keys are signed: a cell of a repeated line adds (n-1) L more in
                    // 32 bits (L - OFF may be negative), clamped at 2^23 - 1 so that
                    // invalid cells stay above every valid one.
                    int key[NJ];
                    if (SPEC && (x == (int)(cxs & 0xFFFFu) || x == (int)(cxs >> 16))) {
                        PairRow<PPL> pr;
#pragma unroll
                        for (int q = 0; q < PPL; q++) pr.v[q] = sv[q];
                        const KeyRow<PPL> kr = corner_keys<PPL>(k.corner, k.side_all, k.H, k.Dp2,
                                                                (int)(k.OFFOFF & 0xFFFFu), y, x, cxs, lane, base_d, pr);
#pragma unroll
                        for (int j = 0; j < NJ; j++) key[j] = kr.v[j];
                    } else {
#pragma unroll
                        for (int q = 0; q < PPL; q++) {
                            key[2 * q] = (int)__byte_perm(sv[q], dpair[q], 0x5104);
                            key[2 * q + 1] = (int)__byte_perm(sv[q], dpair[q], 0x7326);
                        }
                    }
                    int kmin = key[0];
#pragma unroll
                    for (int j = 1; j < NJ; j++) kmin = min(kmin, key[j]);
                    kmin = __reduce_min_sync(FULL, kmin);
                    if (LR) {
                        // logical P[j] (right pixel x - base_d - j) at ring position (T + j) % NJ
#pragma unroll
                        for (int j = 0; j < NJ; j++) P[(T + j) % NJ] = min(P[(T + j) % NJ], key[j]);
                        int in = __shfl_down_sync(FULL, P[N], 1);
                        if (lane == 31) in = INT_MAX;
                        if (lane == 0) {
                            rowR[x] = (uint16_t)(P[N] & 0xFFu);
                            rowL[x] = (uint16_t)(kmin & 0xFFu);
                        }
                        P[N] = in;
                    } else if (lane == 0) {
                        const size_t o = (size_t)y * W + x;
                        const uint16_t dl = (uint16_t)(kmin & 0xFFu);
                        if (k.disp) k.disp[o] = dl;
                        if (k.disp_norm) k.disp_norm[o] = __fdiv_rn((float)dl, (float)k.D);
                    }
                }
                sg += sstep;
                if (zero) return;
#pragma unroll
                for (int q = 0; q < PPL; q++) L[q] = Ln[q];
                m = warp_min_pairs<PPL, EXCL>(L, exm, last_lane);
                if (SPEC && k.GSTART && !started) {
                    // reference GPU recurrence: the second step sees C + P1 with
                    // the minimum of C (tdvision/semiglobal.cu:353-358)
#pragma unroll
                    for (int q = 0; q < PPL; q++) L[q] += k.GSTART;
                }
                if (SPEC) started = true;
            };

            // group j at window positions T0 .. T0+3: wait, run, release its slot
            auto group = [&](auto T0c, int j) -> bool {
                constexpr int T0 = decltype(T0c)::value;
                const int s = j % NSL;
                bool good = chunks_for(j);
                good = good && mbar_wait(fullS(r, s), (uint32_t)(j / NSL) & 1u);
                if (!__all_sync(FULL, good)) return false;
                const unsigned char* slot = wbase + s * SLOT;
                const int xlo = group_lo(j), xhi = group_hi(j), n = xhi - xlo + 1;
                const int cxa = (int)(cxs & 0xFFFFu), cxb = (int)(cxs >> 16);
                const bool special = WTD && ((rflags & 4u) || ((rflags & 2u) && (xlo == 0 || xhi >= W - 1)) ||
                                             (cxa >= xlo && cxa <= xhi) || (cxb >= xlo && cxb <= xhi) ||
                                             (k.GSTART && j == 0));
                if (special) {
                    if constexpr (WTD) {
                        static_for<0, kHpU>([&](auto ic) {
                            constexpr int i = decltype(ic)::value;
                            if (i < n)
                                step(std::integral_constant<int, T0 + i>{}, std::true_type{}, std::true_type{},
                                     DXP ? xlo + i : xhi - i, slot, DXP ? i : n - 1 - i);
                        });
                    }
                } else if (n == kHpU && xlo >= DSPAN && k.D >= DSPAN) {
                    static_for<0, kHpU>([&](auto ic) {
                        constexpr int i = decltype(ic)::value;
                        step(std::integral_constant<int, T0 + i>{}, std::false_type{}, std::false_type{},
                             DXP ? xlo + i : xhi - i, slot, DXP ? i : kHpU - 1 - i);
                    });
                } else {
                    static_for<0, kHpU>([&](auto ic) {
                        constexpr int i = decltype(ic)::value;
                        if (i < n)
                            step(std::integral_constant<int, T0 + i>{}, std::true_type{}, std::false_type{},
                                 DXP ? xlo + i : xhi - i, slot, DXP ? i : n - 1 - i);
                    });
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(emptyS(r, s));
                return true;
            };

            if (!DXP) {
                // walking left the window starts full: entries W - base_d - o
                // (positions of step "x = W"), read once from the padded plane in
                // global memory (the chunk ring only holds what the edge lane
                // loads); entries below 0 belong to masked cells, entry W is
                // dropped before use
                const Plane* rrow = k.RPp + (size_t)y * k.Wp;
#pragma unroll
                for (int o = 0; o < NJ; o++) {
                    const int e = min(max(W - base_d - o, 0), W - 1);
                    const uint4 v = __ldcg((const uint4*)(rrow + e + (e >> 3)));
                    WI[o % NJ] = v.x;
                    WN[o % NJ] = v.y;
                    WX[o % NJ] = v.z;
                }
            }
            constexpr int GPI = 8 / kHpU;  // groups per eight-step iteration
            for (int j = 0; j < ngroups; j += GPI) {
                bool good = true;
                static_for<0, GPI>([&](auto gc) {
                    constexpr int g = decltype(gc)::value;
                    if (good && j + g < ngroups) good = group(std::integral_constant<int, g * kHpU>{}, j + g);
                });
                if (!good) return false;
            }
            return true;
        };

        bool ok;
        if (dx > 0)
            ok = lr ? consume(std::true_type{}, std::true_type{}) : consume(std::true_type{}, std::false_type{});
        else
            ok = lr ? consume(std::false_type{}, std::true_type{}) : consume(std::false_type{}, std::false_type{});
        if (!ok) {
            if (lane == 0) atomicExch(k.err, (int)TDV_ERR_TIMEOUT);
        } else if (lr) {
            __syncwarp();
            for (int xx = lane; xx < W; xx += 32) {
                const int dl = rowL[xx];
                const int xr = xx - dl;
                const bool bad = xr < 0 || abs(dl - (int)rowR[xr]) > k.lr_thr;
                const size_t o = (size_t)y * W + xx;
                if (k.disp) k.disp[o] = bad ? (uint16_t)0xFFFF : (uint16_t)dl;
                if (k.disp_norm) k.disp_norm[o] = bad ? -1.0f : __fdiv_rn((float)dl, (float)k.D);
                if (k.disp_right) k.disp_right[o] = rowR[xx];
            }
        }
    }
    // every role is done with the rings: retire the barriers
    __syncthreads();
    if (threadIdx.x == 0)
        for (int b = 0; b < R * BARS; b++) mbar_inval(smem_u32(&bars[b]));
}

// ------------------------------------------- horizontal passes, split D
// Two warps per image row: warp h owns disparity pairs [h*32*PH, (h+1)*32*PH)
// (PH pairs per lane).  Each step they exchange, through shared memory and one
// 64-thread named barrier, what couples the halves: the minimum of the new L
// (the m of the next step), the boundary neighbour across the split, and in
// the last pass the WTA key and the right-view chain value.  This doubles the
// independent work per SM over one warp per row (1080 rows fill only ~7 warps
// of each of the 148 SMs).
template <int PH, int MODE>
__device__ __forceinline__ void h2_body(const FK& k, int dx, int R, int warp_bytes, int row_bytes, int blk,
                                        unsigned char* smem, bool nc) {
    constexpr int SBH = 128 * PH;  // this warp's share of a pixel's S vector
    constexpr int DH = 64 * PH;    // disparities per warp
    constexpr int NJ = 2 * PH;
    constexpr int CH = kChunk2;  // entries per chunk
    constexpr int CHB = (CH / 8) * kGroupBytes;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ri = warp >> 1, h = warp & 1;
    const int y = blk * R + ri;
    if (ri >= R || y >= k.H) return;  // both warps of the row leave together
    unsigned char* wbase = smem + (size_t)warp * warp_bytes;
    unsigned char* rbase = smem + (size_t)2 * R * warp_bytes + (size_t)ri * row_bytes;
    uint64_t* sbar = (uint64_t*)wbase;
    uint64_t* cbar = sbar + kHSlots;
    unsigned char* sring = wbase + 128;
    unsigned char* cring = sring + kHSlots * SBH;
    uint32_t* xch = (uint32_t*)rbase;  // [2 parity][2 warps][8]
    uint16_t* rowL = (uint16_t*)(rbase + 128);
    uint16_t* rowR = rowL + k.W;
    const bool lr = MODE == 2 && k.lr_thr >= 0;
    const int bar_id = 1 + ri;

    const int W = k.W;
    const int x0 = dx > 0 ? 0 : W - 1;
    const int dlo = h * DH, dhi = dlo + DH;
    const int nch = (W + CH - 1) / CH;
    const int groups_row = (W + 7) / 8;
    const Plane* rrow = k.RPp + (size_t)y * k.Wp;
    const uint32_t* srow = k.S + (size_t)y * W * k.Dp2 + h * (SBH / 4);

    if (lane == 0) {
        for (int b = 0; b < kHSlots + kChunkSlots; b++) mbar_init(smem_u32(&sbar[b]), 1);
        fence_mbar_init();
    }
    __syncwarp();

    auto e_lo = [&](int x) { return max(0, x - dhi + 2); };
    auto e_hi = [&](int x) { return max(0, x - dlo); };
    // a warp walking right to left starts at its own first chunk c0, which is
    // below nch-1 for the upper half; phases count from there
    const int c0 = dx > 0 ? 0 : e_hi(W - 1) / CH;
    auto chunk_use = [&](int c) { return dx > 0 ? c / kChunkSlots : (c0 - c) / kChunkSlots; };
    auto chunk_bar = [&](int c) { return smem_u32(&cbar[c & (kChunkSlots - 1)]); };
    auto issue_chunk = [&](int c) {
        const int ng = min(CH / 8, groups_row - c * (CH / 8));
        const uint32_t bar = chunk_bar(c);
        mbar_expect_tx(bar, (uint32_t)ng * kGroupBytes);
        tma_load(smem_u32(cring + (c & (kChunkSlots - 1)) * CHB), rrow + 9 * (c * (CH / 8)),
                 (uint32_t)ng * kGroupBytes, bar);
    };
    auto issue_s = [&](int t) {
        const int x = x0 + dx * t;
        const uint32_t bar = smem_u32(&sbar[t & (kHSlots - 1)]);
        mbar_expect_tx(bar, SBH);
        tma_load(smem_u32(sring + (t & (kHSlots - 1)) * SBH), srow + (size_t)x * k.Dp2, SBH, bar);
    };

    // chunk window [e_lo(x), e_hi(x)]: `waited` is the last chunk waited for,
    // `next` the next to issue, both moving in the walk direction
    int waited, next;
    if (dx > 0) {
        waited = -1;
        next = 0;
    } else {
        waited = c0 + 1;
        next = c0;
    }
    int s_issued = 0;
    if (lane == 0)
        for (; s_issued < kHSlots && s_issued < W; s_issued++) issue_s(s_issued);
    s_issued = __shfl_sync(FULL, s_issued, 0);

    bool ok = true;
    const int base_d = dlo + lane * 2 * PH;
    const bool edge_lane = base_d + 2 * PH > k.D;
    uint32_t L[PH], m = 0, sv[PH], bnd = k.BIGBIG;
    uint32_t P[NJ];
    #pragma unroll
    for (int j = 0; j < NJ; j++) P[j] = FULL;
    uint4 lp_next = ld_plane(&k.LP[(size_t)y * W + x0], nc);
    uint32_t* sg = k.S + ((size_t)y * W + x0) * k.Dp2 + h * (SBH / 4) + lane * PH;
    const long long sstep = (long long)dx * k.Dp2;

    int t = 0;
    for (; t < W; t++) {
        const int x = x0 + dx * t;
        bool good = true;
        if (dx > 0) {
            const int tc = e_hi(x) / CH;
            if (lane == 0)
                while (next < nch && next <= tc + kLookC) issue_chunk(next++);
            while (good && waited < tc) {
                waited++;
                good = mbar_wait(chunk_bar(waited), (uint32_t)chunk_use(waited) & 1u);
            }
        } else {
            const int tc = e_lo(x) / CH;
            if (lane == 0)
                while (next >= 0 && next >= tc - kLookC) issue_chunk(next--);
            while (good && waited > tc) {
                waited--;
                good = mbar_wait(chunk_bar(waited), (uint32_t)chunk_use(waited) & 1u);
            }
        }
        next = __shfl_sync(FULL, next, 0);
        good = good && mbar_wait(smem_u32(&sbar[t & (kHSlots - 1)]), (uint32_t)(t / kHSlots) & 1u);
        const bool mine_ok = __all_sync(FULL, good);
        uint32_t kmin = FULL;
        if (mine_ok) {
        const uint4 lp = lp_next;
        if (t + 1 < W) lp_next = ld_plane(&k.LP[(size_t)y * W + x + dx], nc);
        uint32_t c[PH], Ln[PH];
        const int eb = x - base_d;
        #pragma unroll
        for (int q = 0; q < PH; q++) {
            const int e = max(eb - 2 * q, 0);
            c[q] = bt_pair(lp, *(const uint4*)(cring + ppos(e & (kChunkSlots * CH - 1)) * 16));
        }
        if (edge_lane || eb < 2 * PH) {
            const int lim = min(x + 1, k.D);
            #pragma unroll
            for (int q = 0; q < PH; q++) c[q] = mask_pair(c[q], base_d + 2 * q, lim, k.BIGBIG);
        }
        if (t == 0) {
            #pragma unroll
            for (int q = 0; q < PH; q++) Ln[q] = c[q];
        } else {
            // neighbours across lanes, and across the two warps at the split
            const uint32_t MM = m * 0x10001u;
            const uint32_t MP2 = MM + k.P2P2;
            uint32_t up = __shfl_up_sync(FULL, L[PH - 1], 1);
            uint32_t dn = __shfl_down_sync(FULL, L[0], 1);
            if (lane == 0) up = h == 0 ? k.BIGBIG : bnd;
            if (lane == 31) dn = h == 1 ? k.BIGBIG : bnd;
            #pragma unroll
            for (int q = 0; q < PH; q++) {
                const uint32_t lm = hi_lo(q > 0 ? L[q - 1] : up, L[q]);
                const uint32_t lpn = hi_lo(L[q], q < PH - 1 ? L[q + 1] : dn);
                uint32_t tv = vmin2(lm, lpn) + k.P1P1;
                tv = vmin2(vmin2(tv, L[q]), MP2);
                Ln[q] = tv + c[q] - MM;
            }
        }
        Vec<PH>::lds((const uint32_t*)(sring + (t & (kHSlots - 1)) * SBH) + lane * PH, sv);
        #pragma unroll
        for (int q = 0; q < PH; q++) sv[q] += Ln[q];
        if (MODE == 1) {
            Vec<PH>::st(sg, sv);
        } else {
            uint32_t key[NJ];
            #pragma unroll
            for (int q = 0; q < PH; q++) {
                key[2 * q] = ((sv[q] & 0xFFFFu) << 8) | (uint32_t)(base_d + 2 * q);
                key[2 * q + 1] = ((sv[q] >> 16) << 8) | (uint32_t)(base_d + 2 * q + 1);
            }
            kmin = key[0];
            #pragma unroll
            for (int j = 1; j < NJ; j++) kmin = min(kmin, key[j]);
            kmin = __reduce_min_sync(FULL, kmin);
            if (lr) {
                #pragma unroll
                for (int j = 0; j < NJ; j++) P[j] = min(P[j], key[j]);
            }
        }
        sg += sstep;
        #pragma unroll
        for (int q = 0; q < PH; q++) L[q] = Ln[q];
        }  // mine_ok
        // ---- exchange with the other half (double-buffered by step parity);
        //      a failed wait on either side ends both warps at this step ----
        uint32_t lmin = L[0];
        #pragma unroll
        for (int q = 1; q < PH; q++) lmin = vmin2(lmin, L[q]);
        lmin = __reduce_min_sync(FULL, min(lmin & 0xFFFFu, lmin >> 16));
        uint32_t* mine = xch + ((t & 1) * 2 + h) * 8;
        const uint32_t* other = xch + ((t & 1) * 2 + (1 - h)) * 8;
        const uint32_t chain_out = __shfl_sync(FULL, P[0], 0);  // warp 1 lane 0 feeds warp 0 lane 31
        const uint32_t edge = __shfl_sync(FULL, h == 0 ? L[PH - 1] : L[0], h == 0 ? 31 : 0);
        if (lane == 0) {
            mine[0] = lmin;
            mine[1] = edge;
            mine[2] = kmin;
            mine[3] = chain_out;
            mine[4] = mine_ok ? 0u : 1u;
        }
        asm volatile("bar.sync %0, 64;" ::"r"(bar_id) : "memory");
        ok = mine_ok && other[4] == 0u;
        if (!ok) break;
        m = min(lmin, other[0]);
        bnd = other[1];
        if (MODE == 2) {
            const uint32_t kk = min(kmin, other[2]);
            if (lr) {
                uint32_t in = __shfl_down_sync(FULL, P[0], 1);
                if (lane == 31) in = h == 0 ? other[3] : FULL;
                if (h == 0 && lane == 0) {
                    rowR[x] = (uint16_t)(P[0] & 0xFFu);
                    rowL[x] = (uint16_t)(kk & 0xFFu);
                }
                #pragma unroll
                for (int j = 0; j < NJ - 1; j++) P[j] = P[j + 1];
                P[NJ - 1] = in;
            } else if (h == 0 && lane == 0) {
                const size_t o = (size_t)y * W + x;
                const uint16_t dl = (uint16_t)(kk & 0xFFu);
                if (k.disp) k.disp[o] = dl;
                if (k.disp_norm) k.disp_norm[o] = __fdiv_rn((float)dl, (float)k.D);
            }
        }
        __syncwarp();
        if (s_issued < W) {
            if (lane == 0) issue_s(s_issued);
            s_issued++;
        }
    }

    if (lane == 0) {
        const uint64_t lim = ok ? kWaitNs : kDrainNs;
        for (int r = t + 1; r < s_issued; r++)
            mbar_wait(smem_u32(&sbar[r & (kHSlots - 1)]), (uint32_t)(r / kHSlots) & 1u, lim);
        if (!ok) mbar_wait(smem_u32(&sbar[t & (kHSlots - 1)]), (uint32_t)(t / kHSlots) & 1u, lim);
        if (dx > 0) {
            for (int c = waited + 1; c < next; c++) mbar_wait(chunk_bar(c), (uint32_t)chunk_use(c) & 1u, lim);
        } else {
            for (int c = waited - 1; c > next; c--) mbar_wait(chunk_bar(c), (uint32_t)chunk_use(c) & 1u, lim);
        }
        if (!ok) atomicExch(k.err, (int)TDV_ERR_TIMEOUT);
        for (int b = 0; b < kHSlots + kChunkSlots; b++) mbar_inval(smem_u32(&sbar[b]));
    }
    if (!ok) return;

    if (lr) {
        asm volatile("bar.sync %0, 64;" ::"r"(bar_id) : "memory");
        for (int xx = h * 32 + lane; xx < W; xx += 64) {
            const int dl = rowL[xx];
            const int xr = xx - dl;
            const bool bad = xr < 0 || abs(dl - (int)rowR[xr]) > k.lr_thr;
            const size_t o = (size_t)y * W + xx;
            if (k.disp) k.disp[o] = bad ? (uint16_t)0xFFFF : (uint16_t)dl;
            if (k.disp_norm) k.disp_norm[o] = bad ? -1.0f : __fdiv_rn((float)dl, (float)k.D);
            if (k.disp_right) k.disp_right[o] = rowR[xx];
        }
    }
}

}  // namespace
}  // namespace tdv
