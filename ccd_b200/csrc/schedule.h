// schedule.h -- dependency-level schedule of one coordinate-descent sweep.
//
// The reference visits coordinates strictly in order j = 0..J-1
// (CyclicCoordinateDescent.cpp:1008-1021); each coordinate reads the row state
// (xBeta, offsExpXBeta, denominators) that earlier coordinates wrote.  Two
// coordinates whose row supports are disjoint (for grouped / Cox models: whose
// stratum sets are disjoint) touch disjoint state, so running them together
// gives exactly the sequential result.  level(j) = 1 + max level of the earlier
// coordinates that touch any row (or stratum) of j; coordinates on one level
// are pairwise disjoint, and running levels in order reproduces the visiting
// order bit for bit.  Each level's columns become tasks (warp / CTA / chunks of
// a long column) statically assigned to the CTAs of a persistent kernel.
#pragma once

#include <cstdint>
#include <vector>

#include "types.h"

namespace ccdb {

struct ScheduleParams {
    int n_cta = 148;          // CTAs of the persistent launch
    int warps_per_cta = 16;   // warps per CTA
    int64_t warp_max = 256;   // columns up to this many entries run on one warp
    int64_t cta_max = 4096;   // ... up to this many on one CTA; longer ones are split
    int64_t chunk = 4096;     // target entries per chunk of a split column
};

struct Schedule {
    int n_cta = 0, n_levels = 0, n_active = 0, n_partials = 0;
    std::vector<int32_t> level_of;   // J, -1 for fixed columns
    std::vector<Task> tasks;
    std::vector<Seg> segs;
    std::vector<int64_t> cta_seg;    // n_cta + 1 offsets into segs
    std::vector<int32_t> level_need; // CTAs active per level
    std::vector<int32_t> col_chunks; // J: number of chunks (0 = not split)
    std::vector<uint8_t> level_split; // n_levels: the level holds a split column
    int64_t max_split_per_seg = 0;
    int64_t max_split_per_level = 0;
};

// key_of_row: the conflict key of each row (row id for independent-row models,
// stratum id for grouped / Cox models).  n_keys: number of distinct keys.
// Column entries: col_start/rows (CSC) for SPARSE/INDICATOR, all rows for
// DENSE/INTERCEPT.  fixed[j]: column not visited.  entries_of[j]: entries a
// column's task walks (nnz, or K for dense-like columns, or the group count).
Schedule build_schedule(int64_t K, int32_t J, const int64_t* col_start, const int32_t* rows,
                        const uint8_t* fmt, const uint8_t* fixed, const int32_t* key_of_row,
                        int64_t n_keys, const int64_t* entries_of, const ScheduleParams& sp);

}  // namespace ccdb
