// spmv_kernels.cuh -- CSR SpMV for sm_100a with pluggable row epilogues.
//
// Replaces spmv_op / fused_spvmv (iterative/BiCGSTAB/spmv.metal:11-132), which
// give one 32-lane SIMD-group to every row (25-27 of 32 lanes idle at 5-7
// nonzeros per row) and use scalar loads.  Here a persistent CTA walks "tiles"
// of consecutive rows holding ~tile_nnz nonzeros (tile boundaries come from a
// binary search of row_ptr, computed once per matrix):
//   1. load phase: the tile's col_ind/values are streamed with coalesced
//      128-bit evict-first loads, x is gathered through the read-only path
//      (x stays L2-resident: the matrix stream is marked evict-first), and the
//      products land in shared memory;
//   2. reduce phase: one thread per row sums its products from shared memory
//      (warp-per-row when the tile's rows are long), then the epilogue runs;
//   3. a tile whose rows exceed the shared capacity takes the block-per-row
//      path (whole CTA strides one long row).
// Epilogues fuse the consumer of A*x (store, dot products, Richardson update,
// FP64 residual) so that no SpMV result makes an extra trip through HBM.
#pragma once
#include <type_traits>
#include <utility>

#include "common.cuh"
#include "internal.hpp"

namespace mps {

// Optional epilogue hooks, detected at compile time:
//   __device__ void begin()         run by every thread once the kernel is
//                                   active (loads the scalars it needs, picks
//                                   buffers by iteration parity);
//   __device__ float gather(int c)  element c of the multiplied vector when it
//                                   is formed from other vectors on the fly
//                                   (x is then unused).
template <class E, class = void> struct epi_has_begin : std::false_type {};
template <class E>
struct epi_has_begin<E, std::void_t<decltype(std::declval<E&>().begin())>> : std::true_type {};
template <class E, class = void> struct epi_has_gather : std::false_type {};
template <class E>
struct epi_has_gather<E, std::void_t<decltype(std::declval<const E&>().gather(0))>> : std::true_type {};

// Epilogues of the solvers keep their scalars in `DevScalars* sc`.  The
// last CTA runs finalize() on a shared-memory copy of them: one cooperative
// load (issued beside the partial sums' loads) instead of a chain of
// dependent global loads by one thread, then the copy is written back.  Only
// block 0's tick() writes the scalars during a launch, before block 0
// arrives, so the copy the last CTA takes is current.
template <class E, class = void> struct epi_has_sc : std::false_type {};
template <class E>
struct epi_has_sc<E, std::enable_if_t<std::is_same<decltype(std::declval<E&>().sc), DevScalars*>::value>>
    : std::true_type {};

template <int NT, class E>
__device__ __forceinline__ void scalars_stage_in(const E& e, DevScalars* sh) {
    if constexpr (epi_has_sc<E>::value) {
        static_assert(sizeof(DevScalars) % 8 == 0, "DevScalars is copied in 8-byte words");
        constexpr int W = (int)(sizeof(DevScalars) / 8);
        const unsigned long long* g = reinterpret_cast<const unsigned long long*>(e.sc);
        unsigned long long* l = reinterpret_cast<unsigned long long*>(sh);
        for (int i = threadIdx.x; i < W; i += NT) l[i] = __ldcg(g + i);
    }
}

// After a block barrier that follows scalars_stage_in.
template <int NT, class E>
__device__ __forceinline__ void finalize_staged(const E& e, const double* tot, DevScalars* sh) {
    if constexpr (epi_has_sc<E>::value) {
        if (threadIdx.x == 0) {
            E ec = e;
            ec.sc = sh;
            ec.finalize(tot);
        }
        __syncthreads();
        constexpr int W = (int)(sizeof(DevScalars) / 8);
        unsigned long long* g = reinterpret_cast<unsigned long long*>(e.sc);
        const unsigned long long* l = reinterpret_cast<const unsigned long long*>(sh);
        for (int i = threadIdx.x; i < W; i += NT) g[i] = l[i];
    } else {
        if (threadIdx.x == 0) e.finalize(tot);
    }
}

template <class E>
__device__ __forceinline__ void epi_begin(E& e) {
    if constexpr (epi_has_begin<E>::value) e.begin();
}
template <class E>
__device__ __forceinline__ float epi_x(const E& e, const float* __restrict__ x, int c) {
    if constexpr (epi_has_gather<E>::value) return e.gather(c);
    else return __ldg(x + c);
}

template <typename T> struct VT;
template <> struct VT<float> { using v4 = float4; };
template <> struct VT<double> { using v4 = double4; };

// Gather helper: x may be FP32 or FP64.
template <typename XT>
__device__ __forceinline__ XT gx(const XT* __restrict__ x, int c) { return __ldg(x + c); }

// Products for 4 consecutive nonzeros [k, k+4) with k % 4 == 0 and all four
// inside the tile, or a masked tail.
template <typename XT, typename ST, bool BF16>
__device__ __forceinline__ void load_prod4(const CsrDev& A, const XT* __restrict__ x, int k,
                                           int k0, int k1, ST* __restrict__ prod) {
    if (k >= k0 && k + 3 < k1) {
        const int4 c = ld_stream(reinterpret_cast<const int4*>(A.ci + k));
        float v0, v1, v2, v3;
        if (BF16) {
            const uint2 raw = __ldcs(reinterpret_cast<const uint2*>(A.vb + k));
            __nv_bfloat162 lo = *reinterpret_cast<const __nv_bfloat162*>(&raw.x);
            __nv_bfloat162 hi = *reinterpret_cast<const __nv_bfloat162*>(&raw.y);
            float2 flo = __bfloat1622float2(lo), fhi = __bfloat1622float2(hi);
            v0 = flo.x; v1 = flo.y; v2 = fhi.x; v3 = fhi.y;
        } else {
            const float4 v = ld_stream(reinterpret_cast<const float4*>(A.v + k));
            v0 = v.x; v1 = v.y; v2 = v.z; v3 = v.w;
        }
        ST* p = prod + (k - k0);
        p[0] = (ST)v0 * (ST)gx(x, c.x);
        p[1] = (ST)v1 * (ST)gx(x, c.y);
        p[2] = (ST)v2 * (ST)gx(x, c.z);
        p[3] = (ST)v3 * (ST)gx(x, c.w);
    } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int kk = k + u;
            if (kk >= k0 && kk < k1) {
                const float v = BF16 ? bf16_to_f(A.vb[kk]) : ld_stream(A.v + kk);
                prod[kk - k0] = (ST)v * (ST)gx(x, ld_stream(A.ci + kk));
            }
        }
    }
}

// Generic tile loop.  Epi must provide:
//   static constexpr int NS;                       number of FP64 sums
//   __device__ void row(int r, ST s, double* acc)  consume row r's A*x
//   __device__ void finalize(const double* tot)    last CTA, thread 0
//   unsigned* counter; double* partials;           (when NS > 0)
// and may provide begin() (no gather(): x is read as given).
template <typename XT, typename ST, bool BF16, class Epi, int NT = kNT>
__global__ void __launch_bounds__(NT, 4)
spmv_tiles(CsrDev A, const XT* __restrict__ x, Epi epi) {
    static_assert(!epi_has_gather<Epi>::value, "spmv_tiles reads x as given");
    extern __shared__ __align__(16) unsigned char spmv_smem[];
    ST* prod = reinterpret_cast<ST*>(spmv_smem);
    __shared__ double red[(Epi::NS > 0 ? Epi::NS : 1) * (NT / 32)];
    __shared__ ST redf[NT / 32];
    __shared__ int last_flag;
    if (blockIdx.x == 0 && threadIdx.x == 0) epi.tick();
    if (!epi.active()) {
        if (blockIdx.x == 0 && threadIdx.x == 0) epi.on_skip();
        return;
    }
    epi_begin(epi);
    double acc[Epi::NS > 0 ? Epi::NS : 1];
#pragma unroll
    for (int i = 0; i < (Epi::NS > 0 ? Epi::NS : 1); ++i) acc[i] = 0.0;

    for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
        const int rs = A.tile_row[t], re = A.tile_row[t + 1];
        if (rs >= re) continue;
        const int k0 = A.rp[rs], k1 = A.rp[re];
        if (k1 - k0 <= A.cap) {
            const int a0 = k0 & ~3;
            const int nvec = (k1 - a0 + 3) >> 2;
            for (int j = threadIdx.x; j < nvec; j += NT)
                load_prod4<XT, ST, BF16>(A, x, a0 + 4 * j, k0, k1, prod);
            __syncthreads();
            const int nrows = re - rs;
            if ((k1 - k0) > 16 * nrows) {
                // long rows: one warp per row
                const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
                for (int r = rs + wid; r < re; r += NT / 32) {
                    const int b = A.rp[r] - k0, e = A.rp[r + 1] - k0;
                    ST s = 0;
                    for (int k = b + lane; k < e; k += 32) s += prod[k];
                    s = warp_sum(s);
                    if (lane == 0) epi.row(r, s, acc);
                }
            } else {
                for (int r = rs + threadIdx.x; r < re; r += NT) {
                    const int b = A.rp[r] - k0, e = A.rp[r + 1] - k0;
                    ST s = 0;
                    for (int k = b; k < e; ++k) s += prod[k];
                    epi.row(r, s, acc);
                }
            }
            __syncthreads();
        } else {
            for (int r = rs; r < re; ++r) {
                const int b = A.rp[r], e = A.rp[r + 1];
                ST s = 0;
                for (int k = b + threadIdx.x; k < e; k += NT) {
                    const float v = BF16 ? bf16_to_f(A.vb[k]) : ld_stream(A.v + k);
                    s += (ST)v * (ST)gx(x, ld_stream(A.ci + k));
                }
                s = block_sum<NT>(s, redf);
                if (threadIdx.x == 0) epi.row(r, s, acc);
            }
        }
    }
    if constexpr (Epi::NS > 0) {
        block_sum_n<NT, Epi::NS>(acc, red);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int i = 0; i < Epi::NS; ++i) epi.partials[i * kMaxPartials + blockIdx.x] = acc[i];
        }
        if (arrive_last(epi.counter, &last_flag)) {
            __shared__ DevScalars s_sc;
            scalars_stage_in<NT>(epi, &s_sc);
            double tot[Epi::NS];
            sum_partials_n<NT, Epi::NS>(epi.partials, kMaxPartials, gridDim.x, red, tot);
            finalize_staged<NT>(epi, tot, &s_sc);
        }
    }
}

// ---- basic epilogues -----------------------------------------------------------
struct EpiStore {
    static constexpr int NS = 0;
    float* y;
    unsigned* counter = nullptr;
    double* partials = nullptr;
    __device__ bool active() const { return true; }
    __device__ void tick() const {}
    __device__ void on_skip() const {}
    __device__ void row(int r, float s, double*) const { y[r] = s; }
    __device__ void finalize(const double*) const {}
};

struct EpiStoreDot {   // y = A x ; *out = w . y
    static constexpr int NS = 1;
    float* y;
    const float* w;
    double* out;
    unsigned* counter;
    double* partials;
    __device__ bool active() const { return true; }
    __device__ void tick() const {}
    __device__ void on_skip() const {}
    __device__ void row(int r, float s, double* acc) const {
        y[r] = s;
        acc[0] += (double)w[r] * (double)s;
    }
    __device__ void finalize(const double* tot) const { *out = tot[0]; }
};

// ||b - A x||^2 in FP64 for an FP32 x: the products of the FP32 values and
// x are exact in FP64 and summed in FP64 (used with ST = double), so this is
// the true residual of the x a solve returns, not its FP32 recurrence.
struct EpiTrueResid {
    static constexpr int NS = 1;
    const float* b;
    double* out;
    unsigned* counter;
    double* partials;
    __device__ bool active() const { return true; }
    __device__ void tick() const {}
    __device__ void on_skip() const {}
    __device__ void row(int r, double s, double* acc) const {
        const double rv = (double)b[r] - s;
        acc[0] += rv * rv;
    }
    __device__ void finalize(const double* tot) const { *out = tot[0]; }
};

// Shared-memory bytes for a tile loop.
template <typename ST>
inline size_t spmv_smem_bytes(const CsrDev& A) { return (size_t)A.cap * sizeof(ST); }

}  // namespace mps
