// schedule_check.cpp -- host fuzz test of build_schedule (ccd_b200/csrc/schedule.cpp),
// built with AddressSanitizer and UndefinedBehaviorSanitizer by
// tests/test_host_sanitizers.py.  Random problems (all four column formats,
// fixed columns, row or stratum keys) under schedule parameters small enough
// that warp, CTA and split-column tasks all occur; every invariant the
// persistent sweep kernel relies on is checked:
//   * level(j) = 1 + max level of the earlier columns sharing a key (dense-like
//     columns conflict with everything), fixed columns have no level;
//   * every active column's tasks cover its entries [0, entries) exactly once,
//     each task in a segment of its column's level;
//   * per CTA, segments in increasing level order, task ranges inside the
//     task array; level_need[L] = CTAs with a segment on level L;
//   * split columns: nchunks = col_chunks[j], partial slots inside n_partials,
//     chunks of one column on distinct CTAs;
//   * the cluster sweep's per-level exchange: level_split[L] is 1 exactly when
//     level L holds a split column, every chunk of a column carries the same
//     slot, and the split columns of one level have distinct slots 0..n-1
//     (n <= max_split_per_level).
// Exit status 0 when every case passes.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <set>
#include <utility>
#include <vector>

#include "schedule.h"

using namespace ccdb;

namespace {

int failures = 0;
long long kinds_seen[3] = {0, 0, 0};  // warp, CTA, split-column tasks checked

void check(bool ok, const char* what, int case_id) {
    if (!ok) {
        if (failures < 20) std::fprintf(stderr, "case %d: %s\n", case_id, what);
        ++failures;
    }
}

void run_case(int case_id, std::mt19937_64& rng) {
    std::uniform_int_distribution<int> kdist(1, 400), jdist(1, 60), fdist(0, 9);
    const int64_t K = kdist(rng);
    const int32_t J = jdist(rng);
    const bool grouped = (rng() % 3) == 0;
    const int64_t n_keys = grouped ? std::max<int64_t>(1, K / (1 + rng() % 8)) : K;
    std::vector<int32_t> key_of_row;
    if (grouped) {  // strata: non-decreasing key per row, as the engine lays rows out
        key_of_row.resize(K);
        for (int64_t k = 0; k < K; ++k) key_of_row[k] = (int32_t)((k * n_keys) / K);
    }
    std::vector<uint8_t> fmt(J), fixed(J);
    std::vector<int64_t> col_start(J + 1, 0), entries(J);
    std::vector<int32_t> rows;
    for (int32_t j = 0; j < J; ++j) {
        const int f = fdist(rng);
        fmt[j] = f == 0 ? F_INTERCEPT : f == 1 ? F_DENSE : f < 6 ? F_SPARSE : F_INDICATOR;
        fixed[j] = (rng() % 7) == 0;
        if (fmt[j] == F_SPARSE || fmt[j] == F_INDICATOR) {
            const double density = std::uniform_real_distribution<double>(0.0, 0.6)(rng);
            for (int64_t k = 0; k < K; ++k)
                if (std::uniform_real_distribution<double>(0.0, 1.0)(rng) < density) rows.push_back((int32_t)k);
        }
        col_start[j + 1] = (int64_t)rows.size();
        entries[j] = (fmt[j] == F_DENSE || fmt[j] == F_INTERCEPT) ? K : col_start[j + 1] - col_start[j];
    }
    ScheduleParams sp;
    sp.n_cta = 1 + (int)(rng() % 9);
    sp.warps_per_cta = 1 + (int)(rng() % 4);
    sp.warp_max = 1 + (int64_t)(rng() % 12);
    sp.cta_max = sp.warp_max + (int64_t)(rng() % 40);
    sp.chunk = 1 + (int64_t)(rng() % 30);
    const Schedule s = build_schedule(K, J, col_start.data(), rows.data(), fmt.data(), fixed.data(),
                                      grouped ? key_of_row.data() : nullptr, n_keys, entries.data(), sp);

    // levels
    std::vector<int32_t> last(n_keys, -1);
    int32_t floor_level = -1, max_level = -1, active = 0;
    for (int32_t j = 0; j < J; ++j) {
        if (fixed[j]) {
            check(s.level_of[j] == -1, "fixed column has a level", case_id);
            continue;
        }
        ++active;
        int32_t want;
        if (fmt[j] == F_DENSE || fmt[j] == F_INTERCEPT) {
            want = max_level + 1;
            floor_level = want;
        } else {
            int32_t m = floor_level;
            for (int64_t p = col_start[j]; p < col_start[j + 1]; ++p) {
                const int64_t key = grouped ? key_of_row[rows[p]] : rows[p];
                m = std::max(m, last[key]);
            }
            want = m + 1;
            for (int64_t p = col_start[j]; p < col_start[j + 1]; ++p)
                last[grouped ? key_of_row[rows[p]] : rows[p]] = want;
        }
        check(s.level_of[j] == want, "level differs from the visiting-order rule", case_id);
        max_level = std::max(max_level, want);
    }
    check(s.n_levels == max_level + 1, "level count", case_id);
    check(s.n_active == active, "active column count", case_id);

    // segments and tasks
    check((int)s.cta_seg.size() == sp.n_cta + 1 && s.cta_seg[0] == 0, "cta_seg offsets", case_id);
    check(s.cta_seg.back() == (int64_t)s.segs.size(), "cta_seg end", case_id);
    std::map<int32_t, std::vector<std::pair<int64_t, int64_t>>> cover;
    std::map<int32_t, std::set<int>> chunk_ctas;
    std::map<int32_t, int32_t> slot_of;                  // split column -> its slot
    std::map<int32_t, std::map<int32_t, int32_t>> level_slots;  // level -> slot -> column
    std::vector<int32_t> need(std::max(0, s.n_levels), 0);
    for (int c = 0; c < sp.n_cta; ++c) {
        int32_t prev = -1;
        for (int64_t q = s.cta_seg[c]; q < s.cta_seg[c + 1]; ++q) {
            const Seg& sg = s.segs[q];
            check(sg.level > prev, "segments of a CTA out of level order", case_id);
            prev = sg.level;
            if (sg.level >= 0 && sg.level < s.n_levels) need[sg.level]++;
            check(sg.n_chunk <= s.max_split_per_seg, "max_split_per_seg", case_id);
            const int64_t n = (int64_t)sg.n_chunk + sg.n_cta + sg.n_warp;
            check(sg.t0 >= 0 && sg.t0 + n <= (int64_t)s.tasks.size(), "segment tasks out of range", case_id);
            if (!(sg.t0 >= 0 && sg.t0 + n <= (int64_t)s.tasks.size())) continue;
            for (int64_t i = 0; i < n; ++i) {
                const Task& t = s.tasks[sg.t0 + i];
                const int kind = i < sg.n_chunk ? 2 : (i < sg.n_chunk + sg.n_cta ? 1 : 0);
                check(t.kind == kind, "task kind order within a segment", case_id);
                check(t.col >= 0 && t.col < J, "task column", case_id);
                if (t.col < 0 || t.col >= J) continue;
                check(s.level_of[t.col] == sg.level, "task on another level's segment", case_id);
                check(0 <= t.p0 && t.p0 <= t.p1 && t.p1 <= entries[t.col], "task entry range", case_id);
                if (kind == 0) check(t.warp >= 0 && t.warp < sp.warps_per_cta, "warp slot", case_id);
                if (kind == 2) {
                    check(t.nchunks == s.col_chunks[t.col], "chunk count", case_id);
                    check(t.chunk >= 0 && t.chunk < t.nchunks, "chunk index", case_id);
                    check(t.part_base >= 0 && t.part_base + t.nchunks <= s.n_partials, "partial slots", case_id);
                    check(chunk_ctas[t.col].insert(c).second, "two chunks of a column on one CTA", case_id);
                    auto it = slot_of.find(t.col);
                    if (it == slot_of.end()) slot_of[t.col] = t.slot;
                    else check(it->second == t.slot, "chunks of a column with different slots", case_id);
                    auto& ls = level_slots[sg.level];
                    auto jt = ls.find(t.slot);
                    if (jt == ls.end()) ls[t.slot] = t.col;
                    else check(jt->second == t.col, "two split columns of a level share a slot", case_id);
                }
                cover[t.col].push_back({t.p0, t.p1});
                kinds_seen[kind]++;
            }
        }
    }
    for (int32_t L = 0; L < s.n_levels; ++L) check(need[L] == s.level_need[L], "level_need", case_id);
    check((int32_t)s.level_split.size() == s.n_levels, "level_split size", case_id);
    for (int32_t L = 0; L < s.n_levels && L < (int32_t)s.level_split.size(); ++L) {
        const auto it = level_slots.find(L);
        const int32_t n = (it == level_slots.end()) ? 0 : (int32_t)it->second.size();
        check(s.level_split[L] == (n > 0 ? 1 : 0), "level_split flag", case_id);
        check(n <= s.max_split_per_level, "max_split_per_level", case_id);
        if (n > 0) check(it->second.rbegin()->first == n - 1 && it->second.begin()->first == 0,
                         "slots of a level are not 0..n-1", case_id);
    }
    for (int32_t j = 0; j < J; ++j) {
        if (fixed[j]) {
            check(cover.count(j) == 0, "task for a fixed column", case_id);
            continue;
        }
        auto& v = cover[j];
        std::sort(v.begin(), v.end());
        int64_t at = 0;
        bool ok = !v.empty();
        for (auto& r : v) {
            ok = ok && r.first == at;
            at = r.second;
        }
        check(ok && at == entries[j], "tasks do not cover the column's entries exactly once", case_id);
    }
}

}  // namespace

// A chain longer than the builder's 16-bit level table holds: 70,000 columns
// that all share row 0 (level j), a dense column in the middle (a level of its
// own that every later column follows), and a fixed column; the builder must
// move to its 32-bit table and keep every level.
void run_long_chain(int case_id) {
    const int32_t J = 70000;
    const int64_t K = 3;
    std::vector<uint8_t> fmt(J, F_INDICATOR), fixed(J, 0);
    std::vector<int64_t> col_start(J + 1, 0), entries(J);
    std::vector<int32_t> rows;
    fmt[40000] = F_DENSE;
    fixed[50000] = 1;
    for (int32_t j = 0; j < J; ++j) {
        if (fmt[j] == F_INDICATOR) rows.push_back(0);
        col_start[j + 1] = (int64_t)rows.size();
        entries[j] = (fmt[j] == F_DENSE) ? K : col_start[j + 1] - col_start[j];
    }
    ScheduleParams sp;
    sp.n_cta = 4;
    sp.warps_per_cta = 4;
    const Schedule s = build_schedule(K, J, col_start.data(), rows.data(), fmt.data(), fixed.data(), nullptr, K,
                                      entries.data(), sp);
    int32_t want = 0;
    bool ok = true;
    for (int32_t j = 0; j < J; ++j) {
        if (fixed[j]) {
            ok = ok && s.level_of[j] == -1;
            continue;
        }
        ok = ok && s.level_of[j] == want;
        ++want;
    }
    check(ok, "levels of a chain beyond the 16-bit table", case_id);
    check(s.n_levels == want, "level count of the long chain", case_id);
}

int main(int argc, char** argv) {
    const int cases = argc > 1 ? std::atoi(argv[1]) : 400;
    std::mt19937_64 rng(12345);
    for (int i = 0; i < cases; ++i) run_case(i, rng);
    run_long_chain(cases);
    if (failures) {
        std::fprintf(stderr, "%d check(s) failed\n", failures);
        return 1;
    }
    std::printf("%d schedules checked: %lld warp, %lld CTA, %lld split-column tasks\n", cases, kinds_seen[0],
                kinds_seen[1], kinds_seen[2]);
    // the parameters must reach every kind of task
    return (kinds_seen[0] > 0 && kinds_seen[1] > 0 && kinds_seen[2] > 0) ? 0 : 2;
}
