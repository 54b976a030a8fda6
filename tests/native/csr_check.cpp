// csr_check.cpp -- host test of build_csr (ccd_b200/csrc/csr_host.cpp), built
// with sanitizers by tests/test_host_sanitizers.py: on random matrices of all
// four column formats, the multi-threaded build (1, 2, 3 and 7 threads, one
// entry per thread at least) must equal a plain one-pass counting sort, entry
// for entry.  Exit status 0 when every case agrees.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "csr_host.h"
#include "types.h"

using namespace ccdb;

int main(int argc, char** argv) {
    const int cases = argc > 1 ? std::atoi(argv[1]) : 200;
    std::mt19937_64 rng(777);
    int failures = 0;
    for (int c = 0; c < cases; ++c) {
        const int64_t K = 1 + rng() % 300;
        const int32_t J = 1 + rng() % 40;
        std::vector<uint8_t> fmt(J);
        std::vector<int64_t> cs(J + 1, 0), vs(J + 1, 0);
        std::vector<int32_t> rows;
        std::vector<double> vals;
        for (int j = 0; j < J; ++j) {
            const int f = rng() % 10;
            fmt[j] = f == 0 ? F_INTERCEPT : f == 1 ? F_DENSE : f < 6 ? F_SPARSE : F_INDICATOR;
            if (fmt[j] == F_DENSE) {
                for (int64_t k = 0; k < K; ++k) vals.push_back((double)(rng() % 1000) / 7.0);
            } else if (fmt[j] != F_INTERCEPT) {
                const unsigned dens = rng() % 100;
                for (int64_t k = 0; k < K; ++k)
                    if (rng() % 100 < dens) {
                        rows.push_back((int32_t)k);
                        if (fmt[j] == F_SPARSE) vals.push_back((double)(rng() % 1000) / 3.0);
                    }
            }
            cs[j + 1] = (int64_t)rows.size();
            vs[j + 1] = (int64_t)vals.size();
        }
        // plain counting sort: rows in order, per row the columns in order
        std::vector<int64_t> ptr(K + 1, 0);
        for (int j = 0; j < J; ++j) {
            if (fmt[j] == F_DENSE || fmt[j] == F_INTERCEPT) {
                for (int64_t k = 0; k < K; ++k) ptr[k + 1]++;
            } else {
                for (int64_t p = cs[j]; p < cs[j + 1]; ++p) ptr[rows[p] + 1]++;
            }
        }
        for (int64_t k = 0; k < K; ++k) ptr[k + 1] += ptr[k];
        std::vector<int32_t> col(ptr[K]);
        std::vector<double> val(ptr[K]);
        std::vector<int64_t> pos(ptr.begin(), ptr.end() - 1);
        for (int j = 0; j < J; ++j) {
            if (fmt[j] == F_DENSE || fmt[j] == F_INTERCEPT) {
                for (int64_t k = 0; k < K; ++k) {
                    const int64_t q = pos[k]++;
                    col[q] = j;
                    val[q] = fmt[j] == F_DENSE ? vals[vs[j] + k] : 1.0;
                }
            } else {
                for (int64_t p = cs[j]; p < cs[j + 1]; ++p) {
                    const int64_t q = pos[rows[p]]++;
                    col[q] = j;
                    val[q] = fmt[j] == F_SPARSE ? vals[vs[j] + (p - cs[j])] : 1.0;
                }
            }
        }
        for (int threads : {1, 2, 3, 7}) {
            const HostCsr h = build_csr(K, J, cs.data(), rows.data(), vs.data(), vals.data(), fmt.data(), threads, 1);
            if (h.row_ptr != ptr || h.col != col || h.val != val) {
                if (failures < 10) std::fprintf(stderr, "case %d, %d threads: differs\n", c, threads);
                ++failures;
            }
        }
    }
    if (failures) return 1;
    std::printf("%d matrices, row-major copies identical for 1, 2, 3, 7 threads\n", cases);
    return 0;
}
