// schedule.cpp -- dependency levels and the static task assignment of a sweep.
#include "schedule.h"

#include <algorithm>
#include <functional>
#include <limits>
#include <numeric>
#include <queue>
#include <stdexcept>

namespace ccdb {

namespace {

bool dense_like(uint8_t f) { return f == F_DENSE || f == F_INTERCEPT; }

}  // namespace

Schedule build_schedule(int64_t K, int32_t J, const int64_t* col_start, const int32_t* rows,
                        const uint8_t* fmt, const uint8_t* fixed, const int32_t* key_of_row,
                        int64_t n_keys, const int64_t* entries_of, const ScheduleParams& sp) {
    Schedule s;
    s.n_cta = sp.n_cta;
    s.level_of.assign(J, -1);
    s.col_chunks.assign(J, 0);

    // ---- levels: level(j) = 1 + max level of earlier columns sharing a key.
    // The table of each key's last level (stored + 1, 0 for none) is 16-bit
    // while the levels fit, which halves its cache footprint, and the walk over
    // a column's keys prefetches the entries it will read; beyond 65,533
    // levels the walk restarts with a 32-bit table.
    int32_t max_level = -1;
    auto levels = [&](auto tag) -> bool {
        using T = decltype(tag);
        const int32_t cap = (int32_t)std::numeric_limits<T>::max() - 1;
        std::vector<T> last(n_keys > 0 ? n_keys : 1, T(0));
        auto key_at = [&](int64_t p) -> int64_t { return key_of_row ? key_of_row[rows[p]] : rows[p]; };
        int32_t floor_level = -1;
        max_level = -1;
        s.n_active = 0;
        for (int32_t j = 0; j < J; ++j) {
            if (fixed && fixed[j]) continue;
            int32_t L;
            if (dense_like(fmt[j])) {
                L = max_level + 1;
                floor_level = L;
            } else {
                const int64_t b = col_start[j], e = col_start[j + 1];
                int32_t m = floor_level + 1;  // (the highest level met) + 1
                for (int64_t p = b; p < e; ++p) {
                    if (p + 24 < e) {
                        if (key_of_row) __builtin_prefetch(&key_of_row[rows[p + 24]]);
                        else __builtin_prefetch(&last[rows[p + 24]]);
                    }
                    const int64_t key = key_at(p);
                    if (key < 0 || key >= n_keys) continue;  // rows outside every group
                    m = std::max<int32_t>(m, (int32_t)last[key]);
                }
                L = m;
                if (L > cap) return false;
                for (int64_t p = b; p < e; ++p) {
                    const int64_t key = key_at(p);
                    if (key < 0 || key >= n_keys) continue;
                    last[key] = (T)(L + 1);
                }
            }
            s.level_of[j] = L;
            max_level = std::max(max_level, L);
            s.n_active++;
        }
        return true;
    };
    if (!levels(uint16_t{})) levels(int32_t{});
    s.n_levels = max_level + 1;

    // columns of each level, in visiting order
    std::vector<int64_t> lvl_start(s.n_levels + 1, 0);
    for (int32_t j = 0; j < J; ++j)
        if (s.level_of[j] >= 0) lvl_start[s.level_of[j] + 1]++;
    std::partial_sum(lvl_start.begin(), lvl_start.end(), lvl_start.begin());
    std::vector<int32_t> lvl_cols(s.n_active);
    {
        std::vector<int64_t> pos(lvl_start.begin(), lvl_start.end() - 1);
        for (int32_t j = 0; j < J; ++j)
            if (s.level_of[j] >= 0) lvl_cols[pos[s.level_of[j]]++] = j;
    }

    const int G = sp.n_cta, W = sp.warps_per_cta;
    const double threads = 32.0 * W;
    // per-CTA list of (level, tasks) built level by level
    std::vector<std::vector<Seg>> cta_segs(G);
    std::vector<std::vector<Task>> cta_tasks(G);
    s.level_need.assign(s.n_levels, 0);

    std::vector<double> load(G);
    std::vector<std::vector<Task>> chunk_t(G), cta_t(G), warp_t(G);
    int rot = 0;
    for (int32_t L = 0; L < s.n_levels; ++L) {
        std::fill(load.begin(), load.end(), 0.0);
        for (int c = 0; c < G; ++c) {
            chunk_t[c].clear();
            cta_t[c].clear();
            warp_t[c].clear();
        }
        std::vector<int32_t> big, mid, small;
        for (int64_t q = lvl_start[L]; q < lvl_start[L + 1]; ++q) {
            const int32_t j = lvl_cols[q];
            const int64_t e = entries_of[j];
            if (e > sp.cta_max) big.push_back(j);
            else if (e > sp.warp_max) mid.push_back(j);
            else small.push_back(j);
        }
        auto by_entries = [&](int32_t a, int32_t b) {
            return entries_of[a] != entries_of[b] ? entries_of[a] > entries_of[b] : a < b;
        };
        std::sort(big.begin(), big.end(), by_entries);
        std::sort(mid.begin(), mid.end(), by_entries);
        std::sort(small.begin(), small.end(), by_entries);

        auto least_loaded = [&](int count) {
            std::vector<int> idx(G);
            for (int c = 0; c < G; ++c) idx[c] = (c + rot) % G;
            std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return load[a] < load[b]; });
            idx.resize(count);
            return idx;
        };
        // split columns: chunks on distinct CTAs
        int32_t slot = 0;
        for (int32_t j : big) {
            const int64_t e = entries_of[j];
            const int C = (int)std::min<int64_t>((e + sp.chunk - 1) / sp.chunk, G);
            s.col_chunks[j] = C;
            auto ctas = least_loaded(C);
            for (int c = 0; c < C; ++c) {
                Task t{};
                t.col = j;
                t.kind = 2;
                t.warp = 0;
                t.chunk = c;
                t.nchunks = C;
                t.part_base = s.n_partials;
                t.p0 = e * c / C;
                t.p1 = e * (c + 1) / C;
                t.slot = slot;
                chunk_t[ctas[c]].push_back(t);
                load[ctas[c]] += (t.p1 - t.p0) / threads + 2.0;
            }
            s.n_partials += C;
            ++slot;
        }
        s.level_split.push_back(slot > 0 ? 1 : 0);
        s.max_split_per_level = std::max<int64_t>(s.max_split_per_level, slot);
        for (int32_t j : mid) {
            auto c = least_loaded(1)[0];
            Task t{};
            t.col = j;
            t.kind = 1;
            t.p0 = 0;
            t.p1 = entries_of[j];
            cta_t[c].push_back(t);
            load[c] += t.p1 / threads + 1.0;
        }
        if (!small.empty()) {
            // pack warp tasks into as few CTAs as their count needs, preferring idle CTAs
            const int m = std::min<int>(G, (int)((small.size() + W - 1) / W));
            auto ctas = least_loaded(m);
            struct Slot {
                double load;
                int cta, warp;
                bool operator>(const Slot& o) const {
                    if (load != o.load) return load > o.load;
                    if (cta != o.cta) return cta > o.cta;
                    return warp > o.warp;
                }
            };
            std::priority_queue<Slot, std::vector<Slot>, std::greater<Slot>> pq;
            for (int c : ctas)
                for (int w = 0; w < W; ++w) pq.push({load[c], c, w});
            for (int32_t j : small) {
                Slot sl = pq.top();
                pq.pop();
                Task t{};
                t.col = j;
                t.kind = 0;
                t.warp = (int16_t)sl.warp;
                t.p0 = 0;
                t.p1 = entries_of[j];
                warp_t[sl.cta].push_back(t);
                sl.load += t.p1 / 32.0 + 1.0;
                pq.push(sl);
            }
        }
        rot = (rot + 17) % G;
        for (int c = 0; c < G; ++c) {
            const size_t n = chunk_t[c].size() + cta_t[c].size() + warp_t[c].size();
            if (n == 0) continue;
            Seg sg{};
            sg.level = L;
            sg.n_chunk = (int32_t)chunk_t[c].size();
            sg.n_cta = (int32_t)cta_t[c].size();
            sg.n_warp = (int32_t)warp_t[c].size();
            sg.t0 = (int64_t)cta_tasks[c].size();
            s.max_split_per_seg = std::max<int64_t>(s.max_split_per_seg, sg.n_chunk);
            cta_tasks[c].insert(cta_tasks[c].end(), chunk_t[c].begin(), chunk_t[c].end());
            cta_tasks[c].insert(cta_tasks[c].end(), cta_t[c].begin(), cta_t[c].end());
            cta_tasks[c].insert(cta_tasks[c].end(), warp_t[c].begin(), warp_t[c].end());
            cta_segs[c].push_back(sg);
            s.level_need[L]++;
        }
    }
    // flatten: task offsets become global
    s.cta_seg.assign(G + 1, 0);
    for (int c = 0; c < G; ++c) {
        const int64_t base = (int64_t)s.tasks.size();
        for (Seg sg : cta_segs[c]) {
            sg.t0 += base;
            s.segs.push_back(sg);
        }
        s.tasks.insert(s.tasks.end(), cta_tasks[c].begin(), cta_tasks[c].end());
        s.cta_seg[c + 1] = (int64_t)s.segs.size();
    }
    return s;
}

}  // namespace ccdb
