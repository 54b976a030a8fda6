// batch_mixed.cu -- the cross-validation grid in mixed precision, with the
// instances of a CTA stepping through the columns in lockstep.
//
// A CTA runs a group of G instances (G = 1, 2 or 4; consecutive in the launch
// order, which sorts by prior variance, so a group's instances need similar
// numbers of sweeps).  Every instance keeps its own weights, coefficients,
// bounds and xBeta and runs the sequential coordinate-descent sweep of a
// standalone fit -- same visiting order, same per-column step -- but the G
// instances visit column j together.  Their row state is interleaved
// instance-minor (xBeta[row][G], FP64), so a gathered row is one 32-byte
// DRAM sector for the whole group at G = 4 instead of one sector per instance,
// and the column's row ids are read once per group.  Each entry's row id
// carries the row's fold in its top bits (row | fold << 24), so the instance
// weight (0 on the held-out fold) costs no extra load.
//
// Precision: the row state xBeta and every coefficient stay FP64.  exp(xBeta),
// the logistic ratio and the per-entry gradient/Hessian terms run in FP32, each
// thread sums its terms with a compensated (two-sum) accumulator, and the
// per-column reduction across threads, the Newton step with its prior and
// bound, the convergence objective and the reported log-likelihoods are FP64.
// The per-entry terms follow Logistic / Poisson incrementGradientAndHessian
// (ModelSpecifics.h:541-568, :1509-1543); the step follows ccdUpdateBeta +
// applyBounds (CyclicCoordinateDescent.cpp:1394-1413, :1503-1520).
//
// Pipeline per column j (one CTA, two barriers), deep enough that no DRAM
// round trip of a later column falls on column j's critical path:
//   * the keys (and values) of column j+4 are copied into shared memory with
//     cp.async (completion is awaited two columns later);
//   * the coefficient, bound and XjY of column j+1 are loaded into registers;
//   * column j's state is gathered into registers, reduced, stepped, and the
//     updated xBeta written back from the same registers.
#include <algorithm>
#include <cstdint>

#include "batch_common.cuh"

namespace ccdb {

namespace {

constexpr int kAhead = 4;          // column j stages column j + kAhead
constexpr int kNBuf = kAhead + 1;  // stage buffers: columns j .. j + kAhead
constexpr int kRing = 8;           // column metadata ring: columns j .. j + kAhead + 1

using namespace bm;

template <int MODEL, int G, int SN>
__global__ void __launch_bounds__(kMT, 1) batch_mixed_kernel(BatchParams P) {
    constexpr int S = Inst<G>::S;    // threads per instance
    constexpr int kE = SN / S;       // staged entries per thread
    __shared__ double s_red2[2][kMW][4][2];
    __shared__ double s_red4[2][kMW][4][4];
    __shared__ double s_xch2[2][4][2];  // cluster exchange of per-CTA sums
    __shared__ double s_xch4[2][4][4];
    __shared__ MMeta s_meta[kRing];
    __shared__ ColXch s_xch;  // per-column exchange of (g, h) between the CTAs of a cluster
    extern __shared__ __align__(16) unsigned char s_dyn[];
    MStage<SN>* st = reinterpret_cast<MStage<SN>*>(s_dyn);

    const int C = P.cluster > 0 ? P.cluster : 1;
    const int rank = (int)(blockIdx.x % C);
    const int n_groups = (P.n_inst + G - 1) / G;
    __shared__ int s_grp;
    __shared__ int s_abv[2];  // per sweep parity: this CTA stopped or saw the abort word
    __shared__ InstCounters s_cnt[4];
    int rb2 = 0, rb4 = 0, xb2 = 0, xb4 = 0;
    unsigned xph = 0;  // parity bits of the exchange slots
    if (threadIdx.x == 0 && C > 1) xch_init(s_xch);

    // Groups come from a queue in launch order (weakest priors first), so the
    // longest fits start first whatever order the clusters are scheduled in.
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) s_grp = atomicAdd(P.queue, 1);
        int grp;
        if (C > 1) {
            cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
            cl.sync();
            grp = *cl.map_shared_rank(&s_grp, 0);
            cl.sync();  // every CTA has read rank 0's slot before any of them leaves or refills it
        } else {
            __syncthreads();
            grp = s_grp;
        }
        if (grp >= n_groups) break;
        const Inst<G> I(P, C, grp, rank);
        const int g = I.g, sl = I.sl, hold = I.hold, J = I.J;
        double* X = I.X;
        inst_setup<G>(P, I, s_red2, rb2, s_xch2, xb2);  // ends with a cluster barrier
        // `late`: this thread's exchange gave up (sums not valid); `aborted`: some
        // CTA's exchange wait ran past its bound.  Either way the group stops
        // stepping but keeps exchanging to the end of the sweep, so every CTA of the
        // cluster takes the same exchanges and barriers; after the sweep's closing
        // cluster barrier every CTA reads the abort word and all leave together.
        bool late = false, aborted = false;
        int sweep_par = 0;

        const int j0 = P.offset_vals ? 1 : 0;
        const bool need_ll = P.conv != C_GRADIENT;
        bool active = I.exists;
        double ll = 0.0;
        double last = inst_objective<MODEL, G>(P, I, active, need_ll, ll, s_red4, rb4, s_xch4, xb4);
        int iteration = 0, flag = R_FAIL;
        if (threadIdx.x < 4) s_cnt[threadIdx.x] = InstCounters{0, 0, 0, 0};
        InstCounters& cnt = s_cnt[g];

        auto stage = [&](int col) {
            const MMeta m = s_meta[col & (kRing - 1)];
            if (!stageable<SN>(m)) return;
            MStage<SN>& b = st[col % kNBuf];
            for (int p = threadIdx.x; p < m.n; p += kMT) {
                cp_async4(&b.k[p], P.keys + m.cb + p);
                if (m.fmt == F_SPARSE) cp_async8(&b.x[p], P.vals + m.vb + p);
            }
        };

        while (__syncthreads_or(active)) {
            // sweep prologue: metadata of the first kAhead + 1 columns, stage the first kAhead
            if (threadIdx.x <= kAhead && j0 + (int)threadIdx.x < J)
                s_meta[(j0 + threadIdx.x) & (kRing - 1)] = I.meta(P, j0 + threadIdx.x);
            __syncthreads();
            for (int q = 0; q < kAhead; ++q)
                if (j0 + q < J) stage(j0 + q);
            cp_async_commit();
            cp_async_wait_all();
            __syncthreads();
            // coefficient, bound, XjY and prior of the next column, one column ahead
            double nb0 = 0.0, nhd0 = 0.0, nxjy0 = 0.0;
            int npt = 0;
            if (j0 < J) {
                if (active) {
                    nb0 = I.Bt[(size_t)j0 * G + g];
                    nhd0 = I.Hd[(size_t)j0 * G + g];
                    nxjy0 = I.Xy[(size_t)j0 * G + g];
                }
                npt = P.ptype[j0];
            }
            long long* tr = (P.trace && blockIdx.x == 0 && threadIdx.x == 0 && iteration == P.trace_sweep)
                                ? P.trace : nullptr;

            for (int j = j0; j < J; ++j) {
                if (tr) tr[6 * j] = clock64();
                // the abort word, read at the start of the column and tested at its end
                const int ab = (I.C > 1 && threadIdx.x == 0) ? ld_volatile_i32(P.abort) : 0;
                const MMeta m = s_meta[j & (kRing - 1)];
                const int n = m.n;
                const bool ind = (m.fmt == F_INDICATOR || m.fmt == F_INTERCEPT);
                const bool staged = stageable<SN>(m);
                const double b0 = nb0, hd0 = nhd0, xjy0 = nxjy0;
                const int pt = npt;
                if (j + 1 < J) {
                    if (active) {
                        nb0 = I.Bt[(size_t)(j + 1) * G + g];
                        nhd0 = I.Hd[(size_t)(j + 1) * G + g];
                        nxjy0 = I.Xy[(size_t)(j + 1) * G + g];
                    }
                    npt = P.ptype[j + 1];
                }
                RawMeta nm{};
                if (threadIdx.x == 0 && j + kAhead + 1 < J) nm = I.raw(P, j + kAhead + 1);
                if (j + kAhead < J) stage(j + kAhead);
                cp_async_commit();
                if (tr) tr[6 * j + 1] = clock64();

                // gather and FP32 terms with compensated sums
                float gs = 0.f, gc = 0.f, hs = 0.f, hc = 0.f;
                double xr[kE];
                const MStage<SN>& c = st[j % kNBuf];
                if (staged) {
                    if (active) {
                        // loads only: every gather of the column is in flight at once
    #pragma unroll
                        for (int i = 0; i < kE; ++i) {
                            const int p = sl + i * S;
                            if (p < n) xr[i] = X[(int64_t)(c.k[p] & kKeyRowMask) * G + g];
                        }
    #pragma unroll
                        for (int i = 0; i < kE; ++i) {
                            const int p = sl + i * S;
                            if (p < n && (c.k[p] >> kKeyRowBits) != hold) {
                                const float x = (m.fmt == F_SPARSE) ? (float)c.x[p] : 1.0f;
                                float gt, ht;
                                entry_terms<MODEL>(xr[i], x, ind, gt, ht);
                                two_sum(gs, gc, gt);
                                two_sum(hs, hc, ht);
                            }
                        }
                    }
                } else if (active) {
                    const bool has_rows = (m.fmt == F_SPARSE || m.fmt == F_INDICATOR);
                    const bool has_vals = (m.fmt == F_SPARSE || m.fmt == F_DENSE);
                    for (int64_t p = sl; p < n; p += S) {
                        const int64_t k = has_rows ? (int64_t)__ldg(P.rows + m.cb + p) : m.cb + p;
                        if (I.held(k)) continue;
                        const float x = has_vals ? (float)__ldg(P.vals + m.vb + p) : 1.0f;
                        float gt, ht;
                        entry_terms<MODEL>(X[k * G + g], x, ind, gt, ht);
                        two_sum(gs, gc, gt);
                        two_sum(hs, hc, ht);
                    }
                }
                double gh[2] = {(double)gs + (double)gc, (double)hs + (double)hc};
                if (tr) tr[6 * j + 2] = clock64();
                group_sum<G, 2>(gh, s_red2, rb2);
                if (I.C > 1 && !xch_sum<G>(I, gh, s_xch, j, xph, (unsigned long long)P.xch_wait_ns, P.abort))
                    late = true;
                if (tr) tr[6 * j + 3] = clock64();

                // the step, computed identically by every thread of the instance
                const double d = (active && !late) ? inst_step<G>(I, j, m.ntot, gh[0], gh[1], b0, hd0, xjy0, pt, cnt)
                                                   : 0.0;
                // update xBeta (FP64) from the gathered registers
                if (d != 0.0) {
                    if (staged) {
    #pragma unroll
                        for (int i = 0; i < kE; ++i) {
                            const int p = sl + i * S;
                            if (p < n) {
                                const double x = (m.fmt == F_SPARSE) ? c.x[p] : 1.0;
                                X[(int64_t)(c.k[p] & kKeyRowMask) * G + g] = xr[i] + d * x;
                            }
                        }
                    } else {
                        const bool has_rows = (m.fmt == F_SPARSE || m.fmt == F_INDICATOR);
                        const bool has_vals = (m.fmt == F_SPARSE || m.fmt == F_DENSE);
                        for (int64_t p = sl; p < n; p += S) {
                            const int64_t k = has_rows ? (int64_t)__ldg(P.rows + m.cb + p) : m.cb + p;
                            const double x = has_vals ? __ldg(P.vals + m.vb + p) : 1.0;
                            X[k * G + g] += d * x;
                        }
                    }
                }
                if (threadIdx.x == 0 && j + kAhead + 1 < J) s_meta[(j + kAhead + 1) & (kRing - 1)] = I.cook(nm);
                if (tr) tr[6 * j + 4] = clock64();
                cp_async_wait_but_last();
                if (__syncthreads_or(late || ab != 0)) {
                    aborted = true;
                    active = false;  // no more steps; the exchanges go on to the sweep's end
                }
                if (tr) tr[6 * j + 5] = clock64();
            }
            cp_async_wait_all();
            if (I.C > 1) {
                // One decision for the whole cluster: every CTA publishes whether it
                // stopped or sees the abort word raised (by any cluster), and after the
                // barrier every CTA ORs the same C values.  Slots alternate by sweep.
                namespace cg = cooperative_groups;
                cg::cluster_group cl = cg::this_cluster();
                if (threadIdx.x == 0) s_abv[sweep_par] = (aborted || ld_volatile_i32(P.abort) != 0) ? 1 : 0;
                cl.sync();
                int any = 0;
                for (int r = 0; r < I.C; ++r) any |= *cl.map_shared_rank(&s_abv[sweep_par], r);
                sweep_par ^= 1;
                aborted = any != 0;
                if (aborted) cl.sync();  // no CTA leaves while a peer still reads its slot
            }
            if (aborted) break;

            if (active) ++iteration;
            const double cur = inst_objective<MODEL, G>(P, I, active, need_ll, ll, s_red4, rb4, s_xch4, xb4);
            if (active) inst_converge(P, cur, last, iteration, flag, active);
        }
        if (aborted) {  // the same decision in every CTA of the cluster: report and leave
            if (I.exists && I.sl == 0 && I.rank == 0) {
                BatchResult r{};
                r.flag = kBatchTimeoutFlag;
                P.results[I.inst] = r;
            }
            return;
        }
        inst_finish<MODEL, G>(P, I, flag, iteration, last, cnt, s_red4, rb4, s_xch4, xb4);
        __syncthreads();
    }  // next group
}

__global__ void batch_keys_kernel(const int32_t* rows, int64_t nnz, const int32_t* fold, int32_t* keys) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = rows[e];
        int32_t f = fold ? fold[k] : -1;
        if (f < 0 || f >= kKeyNoFold) f = kKeyNoFold;
        keys[e] = k | (f << kKeyRowBits);
    }
}

template <int MODEL, int G, int SN>
cudaError_t launch_g(const BatchParams& P, cudaStream_t stream) {
    const size_t smem = sizeof(MStage<SN>) * kNBuf;
    void (*fn)(BatchParams) = batch_mixed_kernel<MODEL, G, SN>;
    static std::atomic<uint64_t> done{0};
    cudaError_t e = once_per_device(done, [&] {
        cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (r != cudaSuccess) return r;
        return cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    if (e != cudaSuccess) return e;
    const int C = P.cluster > 0 ? P.cluster : 1;
    const int n_groups = (P.n_inst + G - 1) / G;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(n_groups * C);
    cfg.blockDim = dim3(kMT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    // as many clusters as can be resident at once (they take groups from the queue)
    int resident = 0;
    e = cudaOccupancyMaxActiveClusters(&resident, fn, &cfg);
    if (e != cudaSuccess) return e;
    if (resident < 1) return cudaErrorInvalidConfiguration;
    cfg.gridDim = dim3(std::min(n_groups, resident) * C);
    return cudaLaunchKernelEx(&cfg, fn, P);
}

template <int MODEL, int G>
cudaError_t launch_sn(const BatchParams& P, cudaStream_t stream) {
    if (P.stage_cap <= 1024)
        return launch_g<MODEL, G, 1024>(P, stream);
    return launch_g<MODEL, G, 3072>(P, stream);
}

template <int MODEL>
cudaError_t launch_m(const BatchParams& P, cudaStream_t stream) {
    switch (P.group) {
    case 1: return launch_sn<MODEL, 1>(P, stream);
    case 2: return launch_sn<MODEL, 2>(P, stream);
    case 4: return launch_sn<MODEL, 4>(P, stream);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_batch_keys(const int32_t* rows, int64_t nnz, const int32_t* fold, int32_t* keys,
                              cudaStream_t stream) {
    if (nnz <= 0) return cudaSuccess;
    batch_keys_kernel<<<148 * 4, 256, 0, stream>>>(rows, nnz, fold, keys);
    return cudaGetLastError();
}

cudaError_t launch_batch_mixed(const BatchParams& P, cudaStream_t stream) {
    return (P.model == M_LOGISTIC) ? launch_m<M_LOGISTIC>(P, stream) : launch_m<M_POISSON>(P, stream);
}

}  // namespace ccdb
