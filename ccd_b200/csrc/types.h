// types.h -- plain data types shared by host code and the CUDA kernels.
#pragma once

#include <cstdint>

namespace ccdb {

// Reference ModelType numbering (src/cyclops/Types.h:134-147).
enum ModelType : int32_t { M_POISSON = 2, M_LOGISTIC = 3, M_CLR = 4, M_CPR = 6, M_COX = 8 };
// FormatType (src/cyclops/CompressedDataMatrix.h:36-38).
enum Fmt : uint8_t { F_DENSE = 0, F_SPARSE = 1, F_INDICATOR = 2, F_INTERCEPT = 3 };
// ConvergenceType (Types.h:108-114) and UpdateReturnFlags (Types.h:124-130).
enum Conv : int32_t { C_GRADIENT = 0, C_LANGE = 1, C_MITTAL = 2 };
enum Flag : int32_t { R_SUCCESS = 0, R_FAIL = 1, R_MAX_ITERATIONS = 2, R_ILLCONDITIONED = 3 };

// Device error codes written into DevStatus::error.
enum DevErr : int32_t { E_NONE = 0, E_WAIT_LEVEL = 1, E_WAIT_COLUMN = 2, E_WAIT_GRID = 3 };

// Work unit of a sweep: one column (or one chunk of a long column).
struct Task {
    int32_t col;
    int16_t kind;  // 0: one warp, 1: one CTA, 2: chunk of a split column (one CTA)
    int16_t warp;  // warp slot for kind 0
    int32_t chunk, nchunks;
    int32_t part_base;  // first partial slot of the split column
    int32_t p0, p1;     // entry range within the column
    int32_t slot;       // split columns: index among the level's split columns
};
static_assert(sizeof(Task) == 32, "Task layout");

// A CTA's share of one dependency level: tasks [t0, t0+n_chunk+n_cta+n_warp)
// ordered chunk tasks, CTA tasks, warp tasks.
struct Seg {
    int32_t level;
    int32_t n_chunk, n_cta, n_warp;
    int64_t t0;
};
static_assert(sizeof(Seg) == 24, "Seg layout");

struct DevStatus {
    int32_t error;       // DevErr
    int32_t error_where; // level / column that timed out
    int32_t flag;        // UpdateReturnFlags of the finished findMode
    int32_t iterations;
    int32_t abort;       // raised by any CTA that gave up waiting
    int32_t pad;
    double objective;
    double last_objective;
    double loglik;
    double log_prior;
    unsigned long long nonzero_steps;  // coordinate steps that moved a coefficient (device sweeps)
    unsigned long long pad2;
};

}  // namespace ccdb
