// noalloc.cu -- a gradient/Hessian entry point that allocates no memory.
//
// Some callers cannot allocate device memory: code running while a CUDA
// stream is being captured into a graph, hosts whose device memory is owned
// by a pool they must not grow, or embedding code given a fixed device
// arena.  For them ccdb_column_gradient_hessian_noalloc computes one column's
// (gradient, Hessian) for an independent-row model (logistic, Poisson) from
// device buffers the caller owns, using only the caller's buffers and a
// fixed scratch array compiled into this library.
//
// The scratch (kNoAllocMaxBlocks per-block partial sums) is a file-scope
// __device__ array: every GPU that loads the library holds it until the
// process exits.  Every call shares it, and it keeps the last call's
// contents; each call overwrites exactly the slots it then reads, so nothing
// needs clearing -- but two calls whose kernels overlap on the GPU (different
// streams, or different host threads on one device) race on it.  The host
// needs the array's device address, which it obtains once per device with
// cudaGetSymbolAddress; the first call on each device does that set-up (no
// allocation) and also loads both models' kernels on that device (with lazy
// module loading a kernel's first launch would otherwise load it then), so
// one call of either model on a device, made before any stream capture
// begins, prepares every later call there.  The address is kept for the life
// of the process: resetting the device (cudaDeviceReset) after that first
// call is not supported.
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/ccdb.h"
#include "common.cuh"

namespace ccdb {

extern thread_local std::string g_last_error;

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxBlocks = 2048;   // scratch slots (32 KiB of double2)
constexpr int64_t kNoAllocPerBlock = 8192;  // entries per block
constexpr int kMaxDevices = 64;

__device__ __align__(256) double2 g_noalloc_partials[kNoAllocMaxBlocks];

double2* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// Per-entry terms of Logistic / Poisson incrementGradientAndHessian
// (ModelSpecifics.h:541-568, :1509-1543) over the row layout
// {xBeta, offsExpXBeta, denominator, weight}.
template <int MODEL>
__global__ void __launch_bounds__(kNoAllocThreads) noalloc_partial_kernel(
    int fmt, int64_t n, const int32_t* rows, const double* vals, const double* state,
    double2* partials) {
    __shared__ double2 s_red[kNoAllocThreads / 32];
    const bool has_rows = (fmt == F_SPARSE || fmt == F_INDICATOR);
    const bool has_vals = (fmt == F_SPARSE || fmt == F_DENSE);
    const bool ind = (fmt == F_INDICATOR || fmt == F_INTERCEPT);
    const int64_t p0 = (int64_t)blockIdx.x * kNoAllocPerBlock;
    const int64_t p1 = (p0 + kNoAllocPerBlock < n) ? p0 + kNoAllocPerBlock : n;
    double g = 0.0, h = 0.0;
    for (int64_t p = p0 + threadIdx.x; p < p1; p += kNoAllocThreads) {
        const int64_t k = has_rows ? (int64_t)rows[p] : p;
        const double x = has_vals ? vals[p] : 1.0;
        const double e = state[4 * k + 1], denom = state[4 * k + 2], w = state[4 * k + 3];
        const double n1 = e * x;
        if (MODEL == M_LOGISTIC) {
            const double gg = n1 / denom;
            g += w * gg;
            if (ind) h += w * gg * (1.0 - gg);
            else h += w * ((n1 * x) / denom - gg * gg);
        } else {
            if (ind) {
                const double v = w * n1;
                g += v;
                h += v;
            } else {
                g += w * n1;
                h += w * (n1 * x);
            }
        }
    }
    const double2 s = block_sum2<kNoAllocThreads / 32>(make_double2(g, h), s_red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void noalloc_finish_kernel(const double2* partials, int nb, int64_t n, double xjy,
                                      double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double2 s = make_double2(0.0, 0.0);
    for (int b = 0; b < nb; ++b) {
        s.x += partials[b].x;
        s.y += partials[b].y;
    }
    // an empty column gives (0, 0) (ModelSpecifics.hpp:720-723)
    out[0] = (n > 0) ? s.x - xjy : 0.0;
    out[1] = (n > 0) ? s.y : 0.0;
}

}  // namespace

}  // namespace ccdb

using namespace ccdb;

extern "C" int ccdb_column_gradient_hessian_noalloc(int32_t model_type, int32_t fmt,
                                                    int64_t n_entries, const int32_t* rows,
                                                    const double* vals, const double* row_state,
                                                    double xjy, double* out, void* stream) {
    auto fail = [](int code, const char* msg) {
        g_last_error = msg;
        return code;
    };
    if (model_type != M_LOGISTIC && model_type != M_POISSON)
        return fail(CCDB_ERR_UNSUPPORTED, "noalloc gradient: logistic and Poisson models only");
    if (fmt < F_DENSE || fmt > F_INTERCEPT || n_entries < 0 || !out || (n_entries > 0 && !row_state))
        return fail(CCDB_ERR_INVALID, "noalloc gradient: bad format, size or NULL buffer");
    if ((fmt == F_SPARSE || fmt == F_INDICATOR) && n_entries > 0 && !rows)
        return fail(CCDB_ERR_INVALID, "noalloc gradient: row ids are required for this format");
    if ((fmt == F_SPARSE || fmt == F_DENSE) && n_entries > 0 && !vals)
        return fail(CCDB_ERR_INVALID, "noalloc gradient: values are required for this format");
    const int64_t nb64 = (n_entries + kNoAllocPerBlock - 1) / kNoAllocPerBlock;
    if (nb64 > kNoAllocMaxBlocks)
        return fail(CCDB_ERR_INVALID,
                    "noalloc gradient: column longer than the fixed scratch allows "
                    "(at most 16,777,216 entries)");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(CCDB_ERR_CUDA, "noalloc gradient: no current CUDA device");
    double2* scratch;
    {
        std::lock_guard<std::mutex> g(g_scratch_mu);
        if (!g_scratch_addr[dev]) {  // once per device, with that device current
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p)
                return fail(CCDB_ERR_CUDA, "noalloc gradient: cannot resolve the scratch address");
            cudaFuncAttributes fa;
            if (cudaFuncGetAttributes(&fa, noalloc_partial_kernel<M_LOGISTIC>) != cudaSuccess ||
                cudaFuncGetAttributes(&fa, noalloc_partial_kernel<M_POISSON>) != cudaSuccess ||
                cudaFuncGetAttributes(&fa, noalloc_finish_kernel) != cudaSuccess)
                return fail(CCDB_ERR_CUDA, "noalloc gradient: cannot load the kernels");
            g_scratch_addr[dev] = static_cast<double2*>(p);
        }
        scratch = g_scratch_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nb = (int)(nb64 > 0 ? nb64 : 1);
    if (n_entries > 0) {
        if (model_type == M_LOGISTIC)
            noalloc_partial_kernel<M_LOGISTIC><<<nb, kNoAllocThreads, 0, s>>>(fmt, n_entries, rows, vals,
                                                                              row_state, scratch);
        else
            noalloc_partial_kernel<M_POISSON><<<nb, kNoAllocThreads, 0, s>>>(fmt, n_entries, rows, vals,
                                                                             row_state, scratch);
    }
    noalloc_finish_kernel<<<1, 32, 0, s>>>(scratch, n_entries > 0 ? nb : 0, n_entries, xjy, out);
    if (cudaGetLastError() != cudaSuccess) return fail(CCDB_ERR_CUDA, "noalloc gradient: launch failed");
    return CCDB_OK;
}
