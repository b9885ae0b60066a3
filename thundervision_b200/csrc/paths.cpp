// Path tables and the pass scheduler for the aggregation kernels.
//
// The reference walks a table of paths one at a time, each forward from its
// start and then backward from its end (tdvision/semiglobalcpu.cpp:210-222;
// the device kernel runs both directions of one path per CTA,
// tdvision/semiglobal.cu:283-466).  Here the same walks are regrouped into
// passes: a pass holds walks of one direction that touch disjoint cells, and
// passes run in an order that gives every cell exactly the sequence of updates
// the sequential loop gives it.  The grouping is computed greedily from the
// sequential walk order with a per-cell "last pass" stamp, so it also covers
// the REF table's stale diagonal ends (repeated reverse walks are merged into
// one walk with a repeat count; a repeat that precedes its own forward walk,
// as in portrait images, lands in an earlier pass).
#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

#include "tdv_internal.hpp"

namespace tdv {

namespace {

struct TableEntry {
    int sx, sy, ex, ey, dx, dy, size;
};

// The descriptor builders of tdvision/semiglobal.cu:116-230 in table order:
// H rows, V columns, (1,1) diagonals from the top edge then the left edge,
// (-1,1) diagonals from the top edge then the right edge.  With `ref` set the
// `end` fields are kept as the reference computes them (for diagonals longer
// than the short image side they are stale); otherwise end = start+(size-1)*dir.
std::vector<TableEntry> make_table(int W, int H, bool ref) {
    std::vector<TableEntry> t;
    const int X1 = W - 1, Y1 = H - 1;
    t.reserve((size_t)3 * (W + H));
    for (int r = 0; r < H; r++) t.push_back({0, r, X1, r, 1, 0, W});
    for (int c = 0; c < W; c++) t.push_back({c, 0, c, Y1, 0, 1, H});
    for (int k = 0; k < W; k++) {
        const int ey = std::min(k, Y1);
        t.push_back({X1 - k, 0, X1, ey, 1, 1, ey + 1});
    }
    for (int k = 1; k < H; k++) {
        const int ex = std::min(Y1 - k, X1);
        t.push_back({0, k, ex, Y1, 1, 1, ex + 1});
    }
    for (int k = 0; k < W; k++) {
        const int n = std::min(k + 1, H);
        t.push_back({k, 0, 0, n - 1, -1, 1, n});
    }
    for (int k = 1; k < H; k++) {
        const int n = std::min(H - k, W);
        t.push_back({X1, k, X1 - n + 1, k + n - 1, -1, 1, n});
    }
    if (!ref)
        for (auto& e : t) {
            e.ex = e.sx + (e.size - 1) * e.dx;
            e.ey = e.sy + (e.size - 1) * e.dy;
        }
    return t;
}

struct PassBuild {
    int dx, dy;
    std::vector<Walk> walks;
};

}  // namespace

bool build_schedule(int W, int H, int table, int paths, PassSchedule& out) {
    out.W = W;
    out.H = H;
    out.table = table;
    out.paths = paths;
    out.passes.clear();
    out.walks.clear();
    const auto tab = make_table(W, H, table == TDV_TABLE_REF);
    std::vector<int32_t> stamp((size_t)W * H, -1);
    std::vector<PassBuild> pb;

    bool ok = true;
    auto inside = [&](int x, int y) { return x >= 0 && x < W && y >= 0 && y < H; };
    auto place = [&](int sx, int sy, int dx, int dy, int len) {
        // every walk is checked against the image before anything indexes it
        if (len < 1 || !inside(sx, sy) || !inside(sx + (len - 1) * dx, sy + (len - 1) * dy)) {
            ok = false;
            return;
        }
        int j0 = 0;
        int x = sx, y = sy;
        for (int i = 0; i < len; i++, x += dx, y += dy)
            j0 = std::max(j0, stamp[(size_t)y * W + x] + 1);
        // A walk identical to one in the latest pass over its cells repeats it.
        if (j0 > 0) {
            PassBuild& last = pb[j0 - 1];
            if (last.dx == dx && last.dy == dy) {
                for (auto it = last.walks.rbegin(); it != last.walks.rend(); ++it)
                    if (it->sx == sx && it->sy == sy && it->len == len) {
                        it->mult++;
                        return;
                    }
            }
        }
        int j = j0;
        while (j < (int)pb.size() && !(pb[j].dx == dx && pb[j].dy == dy)) j++;
        if (j == (int)pb.size()) pb.push_back({dx, dy, {}});
        pb[j].walks.push_back({sx, sy, len, 1, -1});
        x = sx;
        y = sy;
        for (int i = 0; i < len; i++, x += dx, y += dy) stamp[(size_t)y * W + x] = j;
    };

    for (const auto& e : tab) {
        if (paths == 4 && e.dx != 0 && e.dy != 0) continue;
        place(e.sx, e.sy, e.dx, e.dy, e.size);
        place(e.ex, e.ey, -e.dx, -e.dy, e.size);
    }
    out.deferred.clear();
    out.defer_rows = 0;
    for (auto& p : pb) {
        Pass ps;
        ps.dx = p.dx;
        ps.dy = p.dy;
        ps.first = out.walks.size();
        ps.count = p.walks.size();
        ps.dfirst = out.deferred.size();
        ps.dmaxlen = 0;
        long long rows = 0;
        for (size_t i = 0; i < p.walks.size(); i++) {
            Walk& w = p.walks[i];
            if (w.mult <= 1) continue;
            w.defer = (int32_t)rows;
            rows += w.len;
            ps.dmaxlen = std::max(ps.dmaxlen, w.len);
            out.deferred.push_back((int32_t)(ps.first + i));
        }
        ps.dcount = out.deferred.size() - ps.dfirst;
        out.defer_rows = std::max(out.defer_rows, rows);
        out.walks.insert(out.walks.end(), p.walks.begin(), p.walks.end());
        out.passes.push_back(ps);
    }
    return ok;
}

// ------------------------------------------------------------ fused weights
namespace {

// fused direction index of a walk direction (V+ V- D1+ D1- D2+ D2- H+ H-)
int fused_dir(int dx, int dy) {
    if (dx == 0) return dy > 0 ? 0 : 1;
    if (dy == 0) return dx > 0 ? 6 : 7;
    if (dx == dy) return dx > 0 ? 2 : 3;
    return dx < 0 ? 4 : 5;
}
const int kFdx[kFusedDirs] = {0, 0, 1, -1, -1, 1, 1, -1};
const int kFdy[kFusedDirs] = {1, -1, 1, -1, 1, -1, 0, 0};

}  // namespace

bool build_fused_weights(int W, int H, int table, int paths, bool assign, FusedWeights& out, const char** why) {
    auto bad = [&](const char* m) {
        if (why) *why = m;
        return false;
    };
    out = FusedWeights();
    out.W = W;
    out.H = H;
    out.table = table;
    out.paths = paths;
    out.assign = assign ? 1 : 0;
    if (W < 1 || H < 1) return bad("empty image");
    const size_t npx = (size_t)W * H;
    // n[dir][cell]: walks of the direction counted in the cell's final sum,
    // replaying the table's sequential walk order (forward, then backward,
    // per entry; tdvision/semiglobalcpu.cpp:210-222)
    std::vector<uint16_t> n(kFusedDirs * npx, 0);
    const auto tab = make_table(W, H, table == TDV_TABLE_REF);
    auto inside = [&](int x, int y) { return x >= 0 && x < W && y >= 0 && y < H; };
    bool ok = true;
    auto walk = [&](int sx, int sy, int dx, int dy, int len) {
        if (len < 1 || !inside(sx, sy) || !inside(sx + (len - 1) * dx, sy + (len - 1) * dy)) {
            ok = false;
            return;
        }
        const int k = fused_dir(dx, dy);
        const size_t c0 = (size_t)sy * W + sx;
        if (assign)  // the start cell's sum is replaced by this walk's first cost
            for (int j = 0; j < kFusedDirs; j++) n[j * npx + c0] = 0;
        int x = sx, y = sy;
        for (int i = 0; i < len; i++, x += dx, y += dy) {
            uint16_t& v = n[k * npx + (size_t)y * W + x];
            if (v == 0xFFFF) {
                ok = false;
                return;
            }
            v++;
        }
    };
    for (const auto& e : tab) {
        if (paths == 4 && e.dx != 0 && e.dy != 0) continue;
        walk(e.sx, e.sy, e.dx, e.dy, e.size);
        walk(e.ex, e.ey, -e.dx, -e.dy, e.size);
    }
    if (!ok) return bad("a table walk leaves the image");

    auto cls = [](int v) { return v == 0 ? 0 : (v == 1 ? 1 : 2); };
    auto border = [&](int x, int y) { return y == 0 || y == H - 1 || x == 0 || x == W - 1; };
    out.nl = W + H - 1;
    out.nb = 2 * W + 2 * H;
    out.lw_off = 0;
    out.bw_off = (size_t)kFusedDirs * out.nl;
    out.corner_off = (out.bw_off + (size_t)kFusedDirs * out.nb + 15) & ~(size_t)15;
    out.bytes = out.corner_off + (size_t)H * 16;
    out.image.assign(out.bytes, 0);
    unsigned char* lw = out.image.data() + out.lw_off;
    unsigned char* bw = out.image.data() + out.bw_off;
    int32_t* corner = (int32_t*)(out.image.data() + out.corner_off);
    for (int y = 0; y < H; y++) {
        corner[4 * y + 0] = -1;
        corner[4 * y + 2] = -1;
    }
    int corner_line[2] = {INT32_MIN, INT32_MIN};

    for (int k = 0; k < kFusedDirs; k++) {
        const uint16_t* nk = n.data() + k * npx;
        const bool active = paths == 8 || kFdx[k] == 0 || kFdy[k] == 0;
        // border classes, checked against the line classes below
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++)
                if (border(x, y)) bw[(size_t)k * out.nb + border_index(W, H, x, y)] = (unsigned char)cls(nk[(size_t)y * W + x]);
        if (!active) continue;
        // line classes: a line is the set of cells x - s*y = kp (vertical and
        // diagonal) or a row (horizontal).  A line counts in its cells
        // nowhere (0: no walk of the direction takes it), once (1), or once
        // plus a correction from its side rows where a cell counts it n >= 2
        // times (2); border cells may differ (their own classes) under
        // start-assign semantics
        const int dx = kFdx[k], dy = kFdy[k];
        const int s = dx * dy;
        const bool horiz = dy == 0;
        const int nlines = horiz ? H : (s == 0 ? W : W + H - 1);
        const int kmin = s > 0 ? -(H - 1) : 0;
        for (int j = 0; j < nlines; j++) {
            bool any = false, rep = false, in_zero = false, in_pos = false;
            auto visit = [&](int x, int y) {
                const int v = nk[(size_t)y * W + x];
                any |= v > 0;
                rep |= v > 1;
                if (border(x, y)) return;
                (v > 0 ? in_pos : in_zero) = true;
            };
            if (horiz) {
                for (int x = 0; x < W; x++) visit(x, j);
            } else {
                const int kp = kmin + j;
                for (int y = 0; y < H; y++) {
                    const int x = kp + s * y;
                    if (x >= 0 && x < W) visit(x, y);
                }
            }
            if (in_zero && in_pos) return bad("cells inside one path line count it differently");
            if (in_zero && any) return bad("a walked line counts only at the border");
            const int c = rep ? 2 : (any ? 1 : 0);
            if (horiz && rep) return bad("a horizontal line that counts more than once");
            lw[(size_t)k * out.nl + j] = (unsigned char)c;
            if (c != 1) out.has_line = true;
            if (c == 2) {
                const int slot = k == 3 ? 0 : (k == 5 ? 1 : -1);
                if (slot < 0) return bad("a repeated line outside the reverse diagonal directions");
                if (corner_line[slot] != INT32_MIN && corner_line[slot] != j)
                    return bad("two repeated lines in one direction");
                corner_line[slot] = j;
            }
        }
    }
    // border cells, and cells counted more than once
    for (int k = 0; k < kFusedDirs; k++) {
        const uint16_t* nk = n.data() + k * npx;
        const int dx = kFdx[k], dy = kFdy[k], s = dx * dy;
        const int kmin = s > 0 ? -(H - 1) : 0;
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                const int v = nk[(size_t)y * W + x];
                const bool b = border(x, y);
                unsigned char& lc = lw[(size_t)k * out.nl + (dy == 0 ? y : x - s * y - kmin)];
                const int line_cls = lc & 3;
                // the kernels add L on a counted line (class 1 or 2) and the
                // offset alone on a class-0 line; a border cell whose count
                // disagrees takes a class of its own, and its line is flagged
                // (4) so that only flagged lines look border classes up
                if (b && (v == 0) != (line_cls == 0)) {
                    if (!assign) return bad("a border cell that counts unlike its line");
                    out.has_border = true;
                    out.has_line = true;
                    lc |= 4;
                }
                if (v >= 2) {
                    const int slot = k == 3 ? 0 : (k == 5 ? 1 : -1);
                    if (slot < 0 || line_cls != 2) return bad("a repeated cell off the repeated line");
                    int e = corner[4 * y] < 0 ? 0 : 1;
                    if (e == 1 && corner[4 * y + 2] >= 0) return bad("more than two repeated cells in a row");
                    corner[4 * y + 2 * e] = x;
                    corner[4 * y + 2 * e + 1] = ((v - 1) << 1) | slot;
                    out.has_corner = true;
                    out.max_wm1 = std::max(out.max_wm1, v - 1);
                }
            }
    }
    return true;
}

}  // namespace tdv
