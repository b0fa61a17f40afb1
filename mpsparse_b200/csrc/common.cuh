// common.cuh -- shared device helpers for the sm_100a solver kernels.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace mps {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// Device-side error word bits (written with atomicOr, read by the host after
// the stream is synchronised).
enum : unsigned {
    kErrTimeout = 1u,     // a bounded spin gave up
    kErrRange = 2u,       // a COO key was outside the declared shape
    kErrNotFinite = 4u,   // NaN/Inf in a right-hand side
};

// Upper bound on spin iterations of any device-side wait (decoupled look-back,
// mbarrier waits).  With the nanosleep back-off this is well under a second.
constexpr unsigned kSpinLimit = 1u << 22;

// Programmatic dependent launch: a kernel launched with the programmatic
// serialization attribute starts while its predecessor drains and waits here
// until the predecessor has completed and its writes are visible; it then lets
// its own successor begin launching.  Without the attribute both are no-ops.
// Every kernel the solvers launch with the attribute calls this first, before
// touching memory.
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Streaming (evict-first) 128-bit loads for data read exactly once.
__device__ __forceinline__ int4 ld_stream(const int4* p) { return __ldcs(p); }
__device__ __forceinline__ float4 ld_stream(const float4* p) { return __ldcs(p); }
__device__ __forceinline__ int ld_stream(const int* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Deterministic block sum; result valid in thread 0.  `sh` needs NT/32 slots.
template <int NT, typename T>
__device__ __forceinline__ T block_sum(T v, T* sh) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0) sh[w] = v;
    __syncthreads();
    T r = T(0);
    if (threadIdx.x < 32) {
        r = threadIdx.x < NT / 32 ? sh[threadIdx.x] : T(0);
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// Same, but the result is broadcast to every thread.
template <int NT, typename T>
__device__ __forceinline__ T block_sum_all(T v, T* sh) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0) sh[w] = v;
    __syncthreads();
    T r = T(0);
#pragma unroll
    for (int i = 0; i < NT / 32; ++i) r += sh[i];
    __syncthreads();
    return r;
}

// Grid-wide "last block" election after each block published its partial
// result: returns true in every thread of the block that arrived last.  The
// counter is reset by that block so it can be reused by the next launch.
__device__ __forceinline__ bool arrive_last(unsigned* counter, int* sh_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = atomicAdd(counter, 1u);
        *sh_flag = (t == gridDim.x - 1);
    }
    __syncthreads();
    const bool last = *sh_flag != 0;
    if (last) {
        __threadfence();
        if (threadIdx.x == 0) *counter = 0u;
    }
    return last;
}

// Deterministic sum of `count` FP64 partials (fixed order), broadcast.
template <int NT>
__device__ __forceinline__ double sum_partials(const double* part, int count, double* sh) {
    double s = 0.0;
    for (int i = threadIdx.x; i < count; i += NT) s += __ldcg(part + i);
    return block_sum_all<NT>(s, sh);
}

// NS block sums in one pass (one pair of barriers for all of them); the
// same order of additions per sum as block_sum, so the same bits.  sh holds
// NS * NT / 32 values; thread 0 receives the totals.
template <int NT, int NS>
__device__ __forceinline__ void block_sum_n(double (&v)[NS], double* sh) {
    constexpr int W = NT / 32;
    const int w = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NS; ++i) v[i] = warp_sum(v[i]);
    if (lane_id() == 0) {
#pragma unroll
        for (int i = 0; i < NS; ++i) sh[i * W + w] = v[i];
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            const double r = threadIdx.x < W ? sh[i * W + threadIdx.x] : 0.0;
            v[i] = warp_sum(r);
        }
    }
    __syncthreads();
}

// NS sums of `count` FP64 partials each (sum i at part + i * stride), in the
// fixed order of sum_partials, broadcast to every thread.
template <int NT, int NS>
__device__ __forceinline__ void sum_partials_n(const double* part, int stride, int count, double* sh,
                                               double (&tot)[NS]) {
    constexpr int W = NT / 32;
    double s[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) s[i] = 0.0;
    for (int k = threadIdx.x; k < count; k += NT) {
#pragma unroll
        for (int i = 0; i < NS; ++i) s[i] += __ldcg(part + i * stride + k);
    }
    const int w = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NS; ++i) s[i] = warp_sum(s[i]);
    if (lane_id() == 0) {
#pragma unroll
        for (int i = 0; i < NS; ++i) sh[i * W + w] = s[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        double r = 0.0;
#pragma unroll
        for (int j = 0; j < W; ++j) r += sh[i * W + j];
        tot[i] = r;
    }
    __syncthreads();
}

__device__ __forceinline__ float bf16_to_f(__nv_bfloat16 v) { return __bfloat162float(v); }

}  // namespace mps
