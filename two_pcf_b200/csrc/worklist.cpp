// Work-list construction for the pair-count kernels (host side): which runs
// of catalogue B every chunk of catalogue A meets.  Built in parallel over the
// cells of A and concatenated in cell order, so the list does not depend on
// the number of threads.
#include <algorithm>
#include <cstring>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "engine.h"

namespace tpcf {

void decode_cell(const Grid &g, int id, int c[3]) {
    if (g.morton) {
        unsigned v = (unsigned)id;
        for (int m = 0; m < 3; ++m) {
            unsigned x = (v >> m) & 0x09249249u;
            x = (x | (x >> 2)) & 0x030C30C3u;
            x = (x | (x >> 4)) & 0x0300F00Fu;
            x = (x | (x >> 8)) & 0x030000FFu;
            x = (x | (x >> 16)) & 0x3ffu;
            c[m] = (int)x;
        }
    } else {
        c[0] = id / (g.dim[1] * g.dim[2]);
        c[1] = (id / g.dim[2]) % g.dim[1];
        c[2] = id % g.dim[2];
    }
}

int encode_cell(const Grid &g, const int c[3]) {
    for (int m = 0; m < 3; ++m)
        if (c[m] < 0 || c[m] >= g.dim[m]) return -1;
    if (g.morton) {
        unsigned id = 0;
        for (int m = 0; m < 3; ++m) {
            unsigned x = (unsigned)c[m] & 0x3ffu;
            x = (x | (x << 16)) & 0x030000FFu;
            x = (x | (x << 8)) & 0x0300F00Fu;
            x = (x | (x << 4)) & 0x030C30C3u;
            x = (x | (x << 2)) & 0x09249249u;
            id |= x << m;
        }
        return (int)id;
    }
    return (c[0] * g.dim[1] + c[1]) * g.dim[2] + c[2];
}

// Work list.  For every (cell, region) run of A, the segments are the runs
// of B in the cells whose boxes are closer than the maximum separation,
// sorted by region; long A runs are split into chunks of kChunkA points.  For an
// auto count every unordered pair of points is visited once: a B run is a
// segment of an A run when it starts after it in the sorted order, and the A
// run's own segment starts at the chunk and keeps only j > i.
void build_work_items(const Grid &ga, const Grid &gb, bool is_auto, int m, double side, double rb,
                      std::vector<WorkItem> &items, std::vector<Segment> &segs) {
    std::vector<int> offs;
    for (int ox = -m; ox <= m; ++ox)
        for (int oy = -m; oy <= m; ++oy)
            for (int oz = -m; oz <= m; ++oz) {
                double g2 = 0;
                for (int o : {ox, oy, oz}) {
                    double gap = std::max(std::abs(o) - 1, 0) * side * (1.0 - 1e-12);
                    g2 += gap * gap;
                }
                if (g2 < rb * rb) {
                    offs.push_back(ox);
                    offs.push_back(oy);
                    offs.push_back(oz);
                }
            }
    struct Part {
        std::vector<WorkItem> items;
        std::vector<long long> cost;  // A points x B points of each item
        std::vector<Segment> segs;
    };
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    const int nblk = std::max(1, std::min(ga.ncell, 16 * nthreads));
    std::vector<Part> parts(nblk);
#pragma omp parallel for schedule(dynamic, 1)
    for (int blk = 0; blk < nblk; ++blk) {
        const int c0 = (int)((long long)ga.ncell * blk / nblk), c1 = (int)((long long)ga.ncell * (blk + 1) / nblk);
        Part &pt = parts[blk];
        std::vector<Segment> cand;
        for (int ca = c0; ca < c1; ++ca) {
            const int a0 = ga.h_cell_start[ca], a1 = ga.h_cell_start[ca + 1];
            if (a1 == a0) continue;
            int c[3];
            decode_cell(ga, ca, c);
            const int ra0 = ga.h_region_start[ca], ra1 = ga.h_region_start[ca + 1];
            for (int ra = ra0; ra < ra1; ++ra) {
                const int s0 = ga.h_run_start[ra];
                const int s1 = (ra + 1 < ra1) ? ga.h_run_start[ra + 1] : a1;
                cand.clear();
                for (size_t k = 0; k < offs.size(); k += 3) {
                    int cbv[3];
                    for (int mm = 0; mm < 3; ++mm) cbv[mm] = ga.kmin[mm] + c[mm] + offs[k + mm] - gb.kmin[mm];
                    const int cb = encode_cell(gb, cbv);
                    if (cb < 0) continue;
                    const int b0 = gb.h_cell_start[cb], b1 = gb.h_cell_start[cb + 1];
                    if (b1 == b0) continue;
                    if (is_auto && cb < ca) continue;
                    const int rb0 = gb.h_region_start[cb], rb1 = gb.h_region_start[cb + 1];
                    for (int rbk = rb0; rbk < rb1; ++rbk) {
                        const int t0 = gb.h_run_start[rbk];
                        const int t1 = (rbk + 1 < rb1) ? gb.h_run_start[rbk + 1] : b1;
                        if (is_auto && t0 < s0) continue;
                        Segment sg;
                        sg.b_start = t0;
                        sg.b_len = t1 - t0;
                        sg.b_cell = cb;
                        sg.meta = gb.h_regions[rbk] | ((is_auto && t0 == s0) ? (1 << 16) : 0);
                        cand.push_back(sg);
                    }
                }
                if (cand.empty()) continue;
                std::stable_sort(cand.begin(), cand.end(),
                                 [](const Segment &x, const Segment &y) { return (x.meta & 0xffff) < (y.meta & 0xffff); });
                for (int s = s0; s < s1; s += kChunkA) {
                    WorkItem w;
                    std::memset(&w, 0, sizeof(w));
                    w.a_start = s;
                    w.a_len = std::min(kChunkA, s1 - s);
                    w.a_cell = ca;
                    w.a_region = ga.h_regions[ra];
                    w.seg_begin = (int)pt.segs.size();
                    long long bl = 0;
                    for (Segment sg : cand) {
                        if (sg.meta >> 16) {
                            // the A run itself: j > i, starting at this chunk
                            sg.b_len = sg.b_start + sg.b_len - s;
                            sg.b_start = s;
                        }
                        // Close the item when it holds enough B points, so that a
                        // count always splits into many more items than CTAs.
                        if (bl > 0 && bl + sg.b_len > kItemMaxB) {
                            w.seg_end = (int)pt.segs.size();
                            pt.items.push_back(w);
                            pt.cost.push_back((long long)w.a_len * bl);
                            w.seg_begin = (int)pt.segs.size();
                            bl = 0;
                        }
                        bl += sg.b_len;
                        pt.segs.push_back(sg);
                    }
                    w.seg_end = (int)pt.segs.size();
                    pt.items.push_back(w);
                    pt.cost.push_back((long long)w.a_len * bl);
                }
            }
        }
    }
    // Concatenate the parts in block order (in parallel: prefix offsets, then
    // each part copies itself into place).
    std::vector<size_t> io(nblk + 1, 0), so(nblk + 1, 0);
    for (int k = 0; k < nblk; ++k) {
        io[k + 1] = io[k] + parts[k].items.size();
        so[k + 1] = so[k] + parts[k].segs.size();
    }
    const size_t ni = io[nblk];
    std::vector<WorkItem> all(ni);
    std::vector<std::pair<long long, int>> cost(ni);  // (cost, item)
    segs.resize(so[nblk]);
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < nblk; ++k) {
        Part &pt = parts[k];
        const int off = (int)so[k];
        for (size_t q = 0; q < pt.items.size(); ++q) {
            WorkItem w = pt.items[q];
            w.seg_begin += off;
            w.seg_end += off;
            all[io[k] + q] = w;
            cost[io[k] + q] = {pt.cost[q], (int)(io[k] + q)};
        }
        if (!pt.segs.empty()) std::memcpy(segs.data() + so[k], pt.segs.data(), sizeof(Segment) * pt.segs.size());
        std::vector<Segment>().swap(pt.segs);
    }
    // Larger items first (by power-of-two cost class), so the dynamic queue
    // ends balanced; inside a class the items keep the cell order, so the
    // items in flight at once belong to neighbouring cells and share their B
    // tiles in L2 (a full-size s-mu RR count read 104 GB from DRAM in plain
    // longest-first order, 21 GB in this one).
    auto cls = [](long long c) { return c > 0 ? 63 - __builtin_clzll((unsigned long long)c) : -1; };
    std::stable_sort(cost.begin(), cost.end(),
                     [&](const std::pair<long long, int> &x, const std::pair<long long, int> &y) {
                         return cls(x.first) > cls(y.first);
                     });
    items.resize(ni);
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)ni; ++k) items[k] = all[cost[k].second];
}

}  // namespace tpcf
