// mm.h -- the MM algorithm's all-coordinate step (mm.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "types.h"

namespace ccdb {

struct MMParams {
    // CompressedDataMatrix
    const int64_t* col_ptr;
    const int32_t* rows;
    const int64_t* val_ptr;
    const double* vals;
    const uint8_t* fmt;
    int64_t K;
    int32_t J;
    int32_t step;        // 1: also take each free column's step into beta
    // grouped rows: {xBeta, offsExpXBeta}, group of the row; per group: events, denominator
    const double2* xbe;
    const int32_t* grp;
    const double* nEv;
    const double* denom;
    const double* xjy;
    const uint8_t* fixed;  // J flags (nullptr: none)
    // per column
    double* beta;
    const int32_t* ptype;
    const double* pvar;
    double2* gh;           // J outputs {gradient, Hessian bound}
};

// One CTA per column: the MM (gradient, Hessian bound), and with P.step the
// prior's step added to beta (no trust-region bound, as the reference's MM).
cudaError_t launch_mm_gradient_hessian(const MMParams& P, cudaStream_t s);

}  // namespace ccdb
