// Host model of the fused integer-domain path's arithmetic, for the CPU
// tests: BT costs and path costs in 16-bit half-units, the per-direction
// offset and sentinel, the reference CPU recurrence's minimum that leaves out
// d = D-1, the reference GPU recurrence's second step from C + P1, the walk weights of tdv::build_fused_weights (paths.cpp), the
// repeated-line correction and the signed (S << 8 | d) keys of the last pass
// (WTA, right-view disparity, left-right check).  It walks every line of each
// direction once, as the kernels do, and checks every 16-bit value the
// kernels would hold stays in range.
//
// Input file: int32 W, H, D, p1h, p2h, paths, table, semantics, lr_thr, then
// H*W left and H*W right u8 pixels.  Output file: H*W u16 left disparities
// (0xFFFF = rejected by the left-right check), then H*W u16 right-view
// disparities.  Exit status 0 on success, 2 if the weights builder refuses
// the table (the message on stdout), 3 if a value leaves its 16-bit range.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "tdv_internal.hpp"

namespace {

int W, H, D, P1h, P2h, PATHS, TABLE, SEM, LRT;
std::vector<uint8_t> Limg, Rimg;

int px(const std::vector<uint8_t>& im, int x, int y) {
    x = std::min(std::max(x, 0), W - 1);
    y = std::min(std::max(y, 0), H - 1);
    return im[(size_t)y * W + x];
}
void bt_terms(const std::vector<uint8_t>& im, int x, int y, int& i2, int& mn, int& mx) {
    const int v = px(im, x, y), a = v + px(im, x - 1, y), b = v + px(im, x + 1, y);
    i2 = 2 * v;
    mn = std::min(2 * v, std::min(a, b));
    mx = std::max(2 * v, std::max(a, b));
}
// BT in half-units (tdvision/birchfieldcost.cu:14-39), clamp-to-edge taps
int bt(int x, int y, int d) {
    int li, ln, lx, ri, rn, rx;
    bt_terms(Limg, x, y, li, ln, lx);
    bt_terms(Rimg, x - d, y, ri, rn, rx);
    const int A = std::max(li, rn) - std::min(li, rx);
    const int B = std::max(ri, ln) - std::min(ri, lx);
    return std::min(A, B);
}

bool range_error = false;
void check16(long v) {
    if (v < 0 || v > 65535) range_error = true;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) return 1;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 1;
    int32_t hdr[9];
    if (std::fread(hdr, 4, 9, f) != 9) return 1;
    W = hdr[0], H = hdr[1], D = hdr[2], P1h = hdr[3], P2h = hdr[4], PATHS = hdr[5], TABLE = hdr[6], SEM = hdr[7],
    LRT = hdr[8];
    Limg.resize((size_t)W * H);
    Rimg.resize((size_t)W * H);
    if (std::fread(Limg.data(), 1, Limg.size(), f) != Limg.size()) return 1;
    if (std::fread(Rimg.data(), 1, Rimg.size(), f) != Rimg.size()) return 1;
    std::fclose(f);

    const bool excl = SEM == TDV_SEM_REF_CPU;   // min over d < D-1
    const bool assign = SEM == TDV_SEM_REF_CPU;  // start cells restart their sums
    const bool gstart = SEM == TDV_SEM_REF_GPU;  // second step sees C + P1, minimum of C
    tdv::FusedWeights fw;
    const char* why = nullptr;
    const bool weighted = !(TABLE == TDV_TABLE_FULL && !assign);
    if (weighted && !tdv::build_fused_weights(W, H, TABLE, PATHS, assign, fw, &why)) {
        std::printf("weights refused: %s\n", why);
        return 2;
    }
    const int DSPAN = D <= 64 ? 64 : (D <= 128 ? 128 : 256);
    const int OFF = excl ? 510 + std::max(P1h, P2h - P1h) : 0;
    const int BIG = OFF + 511 + 2 * P2h;
    const long KMAX = (1L << 23) - 1;

    // S[cell][d] over the padded disparity span; side[slot][y][d]
    std::vector<long> S((size_t)W * H * DSPAN, 0);
    std::vector<long> side((size_t)2 * H * DSPAN, 0);
    const int fdx[8] = {0, 0, 1, -1, -1, 1, 1, -1}, fdy[8] = {1, -1, 1, -1, 1, -1, 0, 0};
    auto border = [&](int x, int y) { return y == 0 || y == H - 1 || x == 0 || x == W - 1; };
    for (int k = 0; k < 8; k++) {
        const int dx = fdx[k], dy = fdy[k];
        if (PATHS == 4 && dx != 0 && dy != 0) continue;
        const int s = dx * dy, kmin = s > 0 ? -(H - 1) : 0;
        for (int y0 = 0; y0 < H; y0++)
            for (int x0 = 0; x0 < W; x0++) {
                const int px0 = x0 - dx, py0 = y0 - dy;
                if (px0 >= 0 && px0 < W && py0 >= 0 && py0 < H) continue;  // not where a line enters
                int lw = 1;
                if (weighted) lw = fw.image[fw.lw_off + (size_t)k * fw.nl + (dy == 0 ? y0 : x0 - s * y0 - kmin)];
                const int lcls = lw & 3;
                const bool lbw = weighted && fw.has_border && (lw & 4);
                std::vector<long> L(DSPAN, 0), Ln(DSPAN);
                long m = 0;
                bool first = true;
                for (int x = x0, y = y0; x >= 0 && x < W && y >= 0 && y < H; x += dx, y += dy) {
                    long* sc = &S[((size_t)y * W + x) * DSPAN];
                    if (lcls == 0) {  // a line no walk of this direction takes
                        for (int d = 0; d < DSPAN; d++) sc[d] += OFF;
                        continue;
                    }
                    for (int d = 0; d < DSPAN; d++) {
                        const long c = (d <= x && d < D) ? bt(x, y, d) : BIG;
                        const long lm = d > 0 ? L[d - 1] : BIG, lp = d + 1 < DSPAN ? L[d + 1] : BIG;
                        long tv = std::min(lm, lp) + P1h;
                        tv = std::min(std::min(tv, L[d]), m + P2h);
                        Ln[d] = tv + c - m + OFF;
                        check16(Ln[d]);
                    }
                    int cls = lcls;
                    if (lbw && border(x, y))
                        cls = fw.image[fw.bw_off + (size_t)k * fw.nb + tdv::border_index(W, H, x, y)];
                    for (int d = 0; d < DSPAN; d++) {
                        sc[d] += cls == 0 ? OFF : Ln[d];
                        check16(sc[d]);
                    }
                    if (lcls == 2)
                        for (int d = 0; d < DSPAN; d++) side[((size_t)(k == 3 ? 0 : 1) * H + y) * DSPAN + d] = Ln[d];
                    L = Ln;
                    m = LONG_MAX;
                    for (int d = 0; d < DSPAN; d++)
                        if (!(excl && d == D - 1)) m = std::min(m, L[d]);
                    if (gstart && first)
                        for (int d = 0; d < DSPAN; d++) L[d] += P1h;
                    first = false;
                }
            }
    }
    // last pass: keys (S << 8 | d), signed, with the repeated-line correction
    std::vector<uint16_t> dl((size_t)W * H), dr((size_t)W * H);
    const int32_t* corner = weighted ? (const int32_t*)(fw.image.data() + fw.corner_off) : nullptr;
    for (int y = 0; y < H; y++) {
        std::vector<long> P(W, LONG_MAX);
        std::vector<int> rowL(W);
        for (int x = 0; x < W; x++) {
            long best = LONG_MAX;
            for (int d = 0; d < DSPAN; d++) {
                long sv = S[((size_t)y * W + x) * DSPAN + d];
                if (corner)
                    for (int e = 0; e < 2; e++)
                        if (corner[4 * y + 2 * e] == x) {
                            const int code = corner[4 * y + 2 * e + 1];
                            sv += (long)(code >> 1) * (side[((size_t)(code & 1) * H + y) * DSPAN + d] - OFF);
                        }
                sv = std::min(sv, KMAX);
                const long key = sv * 256 + d;
                best = std::min(best, key);
                if (x - d >= 0) P[x - d] = std::min(P[x - d], key);
            }
            rowL[x] = (int)(best & 0xFF);
        }
        for (int x = 0; x < W; x++) {
            const int dL = rowL[x], xr = x - dL;
            const int dR = (int)(P[x] & 0xFF);
            const bool rej = LRT >= 0 && (xr < 0 || std::abs(dL - (int)(P[xr] & 0xFF)) > LRT);
            dl[(size_t)y * W + x] = rej ? 0xFFFF : (uint16_t)dL;
            dr[(size_t)y * W + x] = (uint16_t)dR;
        }
    }
    if (range_error) {
        std::printf("a 16-bit value left its range\n");
        return 3;
    }
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 1;
    std::fwrite(dl.data(), 2, dl.size(), o);
    std::fwrite(dr.data(), 2, dr.size(), o);
    std::fclose(o);
    return 0;
}
