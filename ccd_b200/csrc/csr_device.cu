// csr_device.cu -- the row-major copy of the matrix (computeXBeta's row sums,
// the MM cycle; ModelSpecifics.hpp:313-361 walks the columns per row) built on
// the device from the uploaded column-major arrays.
//
// Pass 1 counts each row's entries (one CTA per column, an atomic add per
// entry: within a column a row appears once), and one CTA turns the counts
// into row offsets (an exclusive scan over tiles of the rows) and finds the
// longest row.  Pass 2 places every entry at its row's cursor (an atomic
// fetch-add; the order inside a row is then the arrival order) and sorts each
// row by column with one thread per row.  A row holds each column at most
// once, so the sorted layout is unique: per row the columns in increasing
// order, the same bytes as the host build (csr_host.cpp) whatever the
// arrival order.  Insertion sort is near linear here because the CTAs of
// pass 2 start in column order.
#include "csr_device.h"

#include <cstdint>

#include "types.h"

namespace ccdb {
namespace {

constexpr int kCT = 256;         // threads of the per-column kernels
constexpr int kST = 1024;        // threads of the scan
constexpr int kSPer = 4;         // rows per scan thread and tile

struct ColRange {
    int64_t cb, vb, n;
    bool has_rows, has_vals;
};

__device__ __forceinline__ ColRange col_range(const CsrDeviceArgs& a, int j) {
    ColRange c;
    const uint8_t f = a.fmt[j];
    c.has_rows = (f == F_SPARSE || f == F_INDICATOR);
    c.has_vals = (f == F_SPARSE || f == F_DENSE);
    c.cb = a.col_ptr[j];
    c.vb = a.val_ptr[j];
    c.n = c.has_rows ? a.col_ptr[j + 1] - c.cb : a.K;
    return c;
}

__global__ void __launch_bounds__(kCT) csr_count_kernel(CsrDeviceArgs a, int32_t* counts) {
    for (int j = blockIdx.x; j < a.J; j += gridDim.x) {
        const ColRange c = col_range(a, j);
        for (int64_t p = threadIdx.x; p < c.n; p += kCT) {
            const int64_t k = c.has_rows ? (int64_t)__ldg(a.rows + c.cb + p) : p;
            atomicAdd(counts + k, 1);
        }
    }
}

// One CTA: tiles of kST * kSPer rows, each thread a run of kSPer rows; the
// thread sums are scanned across the CTA (warp shuffles, then the warp
// totals) and a running carry joins the tiles.
__global__ void __launch_bounds__(kST) csr_scan_kernel(const int32_t* counts, int64_t K, int64_t* row_ptr,
                                                        int64_t* cursor, int32_t* max_row) {
    __shared__ int64_t s_warp[kST / 32];
    __shared__ int64_t s_carry;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) s_carry = 0;
    int32_t longest = 0;
    __syncthreads();
    for (int64_t base = 0; base < K; base += (int64_t)kST * kSPer) {
        const int64_t r0 = base + (int64_t)tid * kSPer;
        int32_t c[kSPer];
        int64_t mine = 0;
#pragma unroll
        for (int i = 0; i < kSPer; ++i) {
            c[i] = (r0 + i < K) ? counts[r0 + i] : 0;
            mine += c[i];
            longest = max(longest, c[i]);
        }
        // inclusive scan of the thread sums within the warp
        int64_t incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) s_warp[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            int64_t w = s_warp[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t v = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += v;
            }
            s_warp[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        const int64_t carry = s_carry;
        int64_t at = carry + (wid > 0 ? s_warp[wid - 1] : 0) + (incl - mine);
#pragma unroll
        for (int i = 0; i < kSPer; ++i)
            if (r0 + i < K) {
                row_ptr[r0 + i] = at;
                cursor[r0 + i] = at;
                at += c[i];
            }
        __syncthreads();  // every thread has read s_carry and s_warp
        if (tid == 0) s_carry = carry + s_warp[kST / 32 - 1];
        __syncthreads();
    }
    // the longest row
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) longest = max(longest, __shfl_xor_sync(0xffffffffu, longest, o));
    __shared__ int32_t s_max[kST / 32];
    if (lane == 0) s_max[wid] = longest;
    __syncthreads();
    if (tid == 0) {
        int32_t m = 0;
        for (int w = 0; w < kST / 32; ++w) m = max(m, s_max[w]);
        *max_row = m;
        row_ptr[K] = s_carry;
    }
}

__global__ void __launch_bounds__(kCT) csr_place_kernel(CsrDeviceArgs a, int64_t* cursor, int32_t* col,
                                                         double* val) {
    for (int j = blockIdx.x; j < a.J; j += gridDim.x) {
        const ColRange c = col_range(a, j);
        for (int64_t p = threadIdx.x; p < c.n; p += kCT) {
            const int64_t k = c.has_rows ? (int64_t)__ldg(a.rows + c.cb + p) : p;
            const double x = c.has_vals ? __ldg(a.vals + c.vb + p) : 1.0;
            const int64_t q = (int64_t)atomicAdd(reinterpret_cast<unsigned long long*>(cursor + k), 1ull);
            col[q] = j;
            val[q] = x;
        }
    }
}

// One thread per row: insertion sort of the row's (column, value) pairs by
// column (columns are distinct within a row).
__global__ void __launch_bounds__(kCT) csr_sort_kernel(const int64_t* row_ptr, int64_t K, int32_t* col,
                                                        double* val) {
    for (int64_t k = (int64_t)blockIdx.x * kCT + threadIdx.x; k < K; k += (int64_t)gridDim.x * kCT) {
        const int64_t lo = row_ptr[k], hi = row_ptr[k + 1];
        for (int64_t i = lo + 1; i < hi; ++i) {
            const int32_t cj = col[i];
            const double vj = val[i];
            int64_t q = i - 1;
            while (q >= lo && col[q] > cj) {
                col[q + 1] = col[q];
                val[q + 1] = val[q];
                --q;
            }
            col[q + 1] = cj;
            val[q + 1] = vj;
        }
    }
}

unsigned col_grid(int32_t J) { return (unsigned)(J < 65535 ? (J > 0 ? J : 1) : 65535); }

}  // namespace

cudaError_t csr_device_count(const CsrDeviceArgs& a, int32_t* counts, int64_t* row_ptr, int64_t* cursor,
                             int32_t* max_row, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int32_t) * (size_t)(a.K > 0 ? a.K : 1), s);
    if (e != cudaSuccess) return e;
    csr_count_kernel<<<col_grid(a.J), kCT, 0, s>>>(a, counts);
    csr_scan_kernel<<<1, kST, 0, s>>>(counts, a.K, row_ptr, cursor, max_row);
    return cudaGetLastError();
}

cudaError_t csr_device_fill(const CsrDeviceArgs& a, const int64_t* row_ptr, int64_t* cursor, int32_t* col,
                            double* val, cudaStream_t s) {
    csr_place_kernel<<<col_grid(a.J), kCT, 0, s>>>(a, cursor, col, val);
    const int64_t blocks = (a.K + kCT - 1) / kCT;
    csr_sort_kernel<<<(unsigned)(blocks < 4096 ? (blocks > 0 ? blocks : 1) : 4096), kCT, 0, s>>>(row_ptr, a.K, col,
                                                                                                  val);
    return cudaGetLastError();
}

}  // namespace ccdb
