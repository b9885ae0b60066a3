// Checks the pass schedule (thundervision_b200/csrc/paths.cpp) for the
// bookkeeping the general SGM passes rely on: every walk lies inside the
// image; the walks of one pass touch disjoint cells; every repeated walk
// (mult > 1) is listed in its pass's deferred range with rows of its own,
// inside PassSchedule::defer_rows; walks that are not repeated have none.
// Prints "schedule: ok" and exits 0 when every size passes.
#include <cstdio>
#include <vector>

#include "tdv_internal.hpp"

static int check(int W, int H, int table, int paths) {
    tdv::PassSchedule sc;
    if (!tdv::build_schedule(W, H, table, paths, sc)) {
        std::printf("%dx%d table %d paths %d: build failed\n", W, H, table, paths);
        return 1;
    }
    std::vector<int> seen((size_t)W * H);
    for (size_t p = 0; p < sc.passes.size(); p++) {
        const tdv::Pass& ps = sc.passes[p];
        std::fill(seen.begin(), seen.end(), 0);
        std::vector<int> rows((size_t)(sc.defer_rows > 0 ? sc.defer_rows : 1), 0);
        size_t repeated = 0;
        for (size_t i = ps.first; i < ps.first + ps.count; i++) {
            const tdv::Walk& w = sc.walks[i];
            for (int t = 0; t < w.len; t++) {
                const int x = w.sx + t * ps.dx, y = w.sy + t * ps.dy;
                if (x < 0 || x >= W || y < 0 || y >= H) return std::printf("walk outside\n"), 1;
                if (seen[(size_t)y * W + x]++) return std::printf("pass %zu: cells shared\n", p), 1;
            }
            if (w.mult > 1) {
                repeated++;
                if (w.defer < 0 || w.defer + w.len > sc.defer_rows) return std::printf("defer range\n"), 1;
                for (int t = 0; t < w.len; t++)
                    if (rows[(size_t)w.defer + t]++) return std::printf("pass %zu: defer rows shared\n", p), 1;
                bool listed = false;
                for (size_t k = ps.dfirst; k < ps.dfirst + ps.dcount; k++) listed |= sc.deferred[k] == (int)i;
                if (!listed) return std::printf("pass %zu: repeated walk not listed\n", p), 1;
            } else if (w.defer != -1) {
                return std::printf("pass %zu: plain walk with deferred rows\n", p), 1;
            }
        }
        if (repeated != ps.dcount) return std::printf("pass %zu: deferred count\n", p), 1;
    }
    return 0;
}

int main() {
    const int sizes[][2] = {{1, 1}, {2, 5}, {5, 2}, {17, 3}, {3, 17}, {64, 48}, {96, 64}, {200, 37}, {37, 200}};
    int bad = 0;
    for (const auto& s : sizes)
        for (int table = 0; table < 2; table++)
            for (int paths : {4, 8}) bad += check(s[0], s[1], table, paths);
    std::printf(bad ? "schedule: FAILED\n" : "schedule: ok\n");
    return bad ? 1 : 0;
}
