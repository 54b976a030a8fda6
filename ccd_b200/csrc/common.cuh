// common.cuh -- device-side building blocks shared by the sweep kernels:
// data descriptors, the Newton/prior/bound step, reductions, and bounded
// inter-CTA synchronisation (every wait has an iteration cap and sets an error
// word instead of hanging).
#pragma once

#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "types.h"
#include "step.h"

namespace ccdb {

// ---------------------------------------------------------------- host: attributes
// A kernel's function attributes (dynamic shared memory, cluster size) are set
// once per device, at its first launch, not before every launch: fits on
// other streams launch the same kernels concurrently.
template <typename F>
inline cudaError_t once_per_device(std::atomic<uint64_t>& done, F&& set) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = set();
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

__device__ __forceinline__ double4 warp_sum4(double4 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        v.z += __shfl_xor_sync(0xffffffffu, v.z, o);
        v.w += __shfl_xor_sync(0xffffffffu, v.w, o);
    }
    return v;
}

// Block-wide sum with a fixed combination order (deterministic).  scratch
// holds one double2 per warp.  Result valid in every thread.
template <int NWARPS>
__device__ __forceinline__ double2 block_sum2(double2 v, double2* scratch) {
    v = warp_sum2(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    double2 t = make_double2(0.0, 0.0);
#pragma unroll
    for (int w = 0; w < NWARPS; ++w) {
        t.x += scratch[w].x;
        t.y += scratch[w].y;
    }
    __syncthreads();
    return t;
}

template <int NWARPS>
__device__ __forceinline__ double4 block_sum4(double4 v, double4* scratch) {
    v = warp_sum4(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    double4 t = make_double4(0.0, 0.0, 0.0, 0.0);
#pragma unroll
    for (int w = 0; w < NWARPS; ++w) {
        t.x += scratch[w].x;
        t.y += scratch[w].y;
        t.z += scratch[w].z;
        t.w += scratch[w].w;
    }
    __syncthreads();
    return t;
}

// ---------------------------------------------------------------- sync
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_gpu_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile_i32(const int32_t* p) {
    return *reinterpret_cast<const volatile int32_t*>(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Spin (one thread) until *p >= target (wrap-safe), or give up once `limit_ns`
// nanoseconds have passed or another CTA has raised st->abort.  Returns true
// on success.  On timeout the caller's error code is recorded and abort is
// raised so every CTA unwinds instead of waiting forever.
__device__ __forceinline__ bool wait_geq(const unsigned* p, unsigned target, long long limit_ns,
                                         DevStatus* st, int err, int where) {
    if ((int)(ld_acquire_gpu(p) - target) >= 0) return true;
    const unsigned long long t0 = global_ns();
    unsigned n = 0;
    while ((int)(ld_acquire_gpu(p) - target) < 0) {
        ++n;
        if (n == 1 || (n & 63) == 0) {  // the first look, then every 64th
            if (ld_volatile_i32(&st->abort)) return false;
            if ((long long)(global_ns() - t0) > limit_ns) {
                if (atomicCAS(&st->error, 0, err) == 0) st->error_where = where;
                atomicExch(&st->abort, 1);
                __threadfence();
                return false;
            }
        }
        if (n > 32) __nanosleep(20);
    }
    return true;
}

// Counter-based grid barrier over all CTAs of a co-resident (cooperative)
// launch.  `epoch` is the caller's running count of barriers passed.
__device__ __forceinline__ bool grid_barrier(unsigned* counter, unsigned& epoch, long long limit,
                                             DevStatus* st, int32_t* s_fail) {
    __syncthreads();
    if (threadIdx.x == 0) {
        ++epoch;
        // the CTA's writes, ordered before this thread's by the barrier above, are
        // released with the arrival; the waits' acquire loads order every later read
        red_release_gpu_add(counter, 1u);
        const bool ok = wait_geq(counter, epoch * gridDim.x, limit, st, E_WAIT_GRID, -1);
        *s_fail = ok ? 0 : 1;
    }
    __syncthreads();
    return *s_fail == 0;
}

}  // namespace ccdb
