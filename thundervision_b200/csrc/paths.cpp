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

}  // namespace tdv
