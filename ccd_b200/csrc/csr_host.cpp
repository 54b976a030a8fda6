// csr_host.cpp -- multi-threaded build of the row-major copy used to recompute
// xBeta from beta (warm starts, the MM cycle).  Columns are split into T
// contiguous ranges of about equal entry counts; thread t counts its range's
// entries per row, the per-row counts turn into each thread's first slot in
// every row (rows in order, threads in order within a row), and each thread
// then places its entries in column order.  Entries of a row therefore keep
// increasing column order whatever T is.
#include "csr_host.h"

#include <algorithm>
#include <system_error>
#include <thread>

#include "types.h"

namespace ccdb {
namespace {

bool dense_like(uint8_t f) { return f == F_DENSE || f == F_INTERCEPT; }

template <typename F>
void run_parallel(int T, F&& f) {
    if (T <= 1) {
        f(0);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(T);
    int started = 0;
    try {
        for (; started < T; ++started) pool.emplace_back(f, started);
    } catch (const std::system_error&) {  // no more threads: this one runs the rest
        for (int t = started; t < T; ++t) f(t);
    }
    for (auto& th : pool) th.join();
}

}  // namespace

HostCsr build_csr(int64_t K, int32_t J, const int64_t* col_start, const int32_t* rows,
                  const int64_t* val_start, const double* vals, const uint8_t* fmt, int threads,
                  int64_t min_per_thread) {
    auto entries = [&](int j) -> int64_t {
        return dense_like(fmt[j]) ? K : col_start[j + 1] - col_start[j];
    };
    int64_t total = 0;
    for (int j = 0; j < J; ++j) total += entries(j);
    // small matrices: one thread (thread start-up would dominate); the count and
    // slot tables (12 bytes per row per thread) stay under 256 MiB
    const int64_t by_work = total / std::max<int64_t>(1, min_per_thread);
    const int64_t by_memory = (int64_t(256) << 20) / std::max<int64_t>(1, 12 * K);
    int T = (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)threads, by_work, by_memory, 64}));
    // column ranges [lo[t], lo[t+1]) of about total / T entries each
    std::vector<int32_t> lo(T + 1, J);
    lo[0] = 0;
    {
        int64_t acc = 0;
        int t = 1;
        for (int j = 0; j < J && t < T; ++j) {
            acc += entries(j);
            if (acc >= total * t / T) lo[t++] = j + 1;
        }
        for (; t < T; ++t) lo[t] = J;
    }
    std::vector<std::vector<int32_t>> cnt(T);
    run_parallel(T, [&](int t) {
        std::vector<int32_t>& c = cnt[t];
        c.assign(K, 0);
        for (int j = lo[t]; j < lo[t + 1]; ++j) {
            if (dense_like(fmt[j])) {
                for (int64_t k = 0; k < K; ++k) c[k]++;
            } else {
                for (int64_t p = col_start[j]; p < col_start[j + 1]; ++p) c[rows[p]]++;
            }
        }
    });
    HostCsr out;
    out.row_ptr.assign(K + 1, 0);
    std::vector<std::vector<int64_t>> slot(T, std::vector<int64_t>(K));
    for (int64_t k = 0; k < K; ++k) {  // rows in order, threads in order within a row
        int64_t at = out.row_ptr[k];
        for (int t = 0; t < T; ++t) {
            slot[t][k] = at;
            at += cnt[t][k];
        }
        out.row_ptr[k + 1] = at;
    }
    cnt.clear();
    out.col.resize(total);
    out.val.resize(total);
    run_parallel(T, [&](int t) {
        std::vector<int64_t>& s = slot[t];
        for (int j = lo[t]; j < lo[t + 1]; ++j) {
            const uint8_t f = fmt[j];
            if (dense_like(f)) {
                for (int64_t k = 0; k < K; ++k) {
                    const int64_t q = s[k]++;
                    out.col[q] = j;
                    out.val[q] = (f == F_DENSE) ? vals[val_start[j] + k] : 1.0;
                }
            } else {
                for (int64_t p = col_start[j]; p < col_start[j + 1]; ++p) {
                    const int64_t q = s[rows[p]]++;
                    out.col[q] = j;
                    out.val[q] = (f == F_SPARSE) ? vals[val_start[j] + (p - col_start[j])] : 1.0;
                }
            }
        }
    });
    return out;
}

}  // namespace ccdb
