// bcsr_kernels.cuh -- BCSR SpMV (4x4 / 8x8 row-major blocks) for sm_100a.
//
// Replaces spmv_op / fused_spvmv of iterative/BiCGSTAB/bcsr_spmv.metal:30-138,
// which gives one thread to a whole block row and reads the block values with
// uncoalesced float4 loads.  Here a persistent CTA walks tiles of consecutive
// block rows.  A tile's block values are one contiguous byte range, so one
// thread stages it into shared memory with a bulk async copy
// (cp.async.bulk, completion on an mbarrier; no multicast), double-buffered so
// the next tile streams in while this one is multiplied.  One thread then owns
// one scalar row: it reads its B-wide row of every block from shared memory
// and the matching x segment (float4 gathers, L2-resident), and hands the sum
// to the same epilogues as the CSR kernel.  All mbarrier waits are bounded.
#pragma once
#include "common.cuh"
#include "internal.hpp"
#include "tma.cuh"
#include "spmv_kernels.cuh"

namespace mps {

struct BcsrDev {
    const int* rp;          // block row_ptr [nbr + 1]
    const int* ci;          // block col_ind [nb]
    const float* v;         // nb * B * B
    const int* tile_brow;   // ntiles + 1 block-row boundaries
    int nbr;
    int ntiles;
    int cap_blocks;         // staged blocks per buffer
    unsigned* err;
};

// Row k of block j times the x segment: B-wide dot product.
template <int B>
__device__ __forceinline__ float block_row_dot(const float* __restrict__ row,
                                               const float* __restrict__ x, int bc) {
    const float4* r4 = reinterpret_cast<const float4*>(row);
    const float4* x4 = reinterpret_cast<const float4*>(x + (size_t)bc * B);
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < B / 4; ++q) {
        const float4 a = r4[q];
        const float4 b = __ldg(x4 + q);
        s = fmaf(a.x, b.x, s);
        s = fmaf(a.y, b.y, s);
        s = fmaf(a.z, b.z, s);
        s = fmaf(a.w, b.w, s);
    }
    return s;
}

template <int B, class Epi, int NT = kNT>
__global__ void __launch_bounds__(NT, 2)
bcsr_tiles(BcsrDev A, const float* __restrict__ x, Epi epi) {
    extern __shared__ __align__(128) unsigned char bcsr_smem[];
    __shared__ unsigned long long bar[2];
    __shared__ double red[(Epi::NS > 0 ? Epi::NS : 1) * (NT / 32)];
    __shared__ int last_flag;
    __shared__ int timed_out;
    if (blockIdx.x == 0 && threadIdx.x == 0) epi.tick();
    if (!epi.active()) {
        if (blockIdx.x == 0 && threadIdx.x == 0) epi.on_skip();
        return;
    }
    constexpr int BB = B * B;
    float* buf[2] = {reinterpret_cast<float*>(bcsr_smem),
                     reinterpret_cast<float*>(bcsr_smem) + (size_t)A.cap_blocks * BB};
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        timed_out = 0;
        fence_mbar_init();
    }
    __syncthreads();
    double acc[Epi::NS > 0 ? Epi::NS : 1];
#pragma unroll
    for (int i = 0; i < (Epi::NS > 0 ? Epi::NS : 1); ++i) acc[i] = 0.0;

    unsigned uses0 = 0u, uses1 = 0u;   // completed phases per buffer (uniform)   // completed phases per buffer (uniform)
    auto staged = [&](int t) {
        const int j0 = A.rp[A.tile_brow[t]], j1 = A.rp[A.tile_brow[t + 1]];
        return j1 - j0 <= A.cap_blocks && j1 > j0;
    };
    auto issue = [&](int t, int b) {   // thread 0 only
        const int j0 = A.rp[A.tile_brow[t]], j1 = A.rp[A.tile_brow[t + 1]];
        const unsigned bytes = (unsigned)(j1 - j0) * BB * sizeof(float);
        fence_proxy_async();
        mbar_expect_tx(&bar[b], bytes);
        bulk_g2s(buf[b], A.v + (size_t)j0 * BB, bytes, &bar[b]);
    };
    int it = 0;
    int t = blockIdx.x;
    if (t < A.ntiles && threadIdx.x == 0 && staged(t)) issue(t, 0);
    for (; t < A.ntiles; t += gridDim.x, ++it) {
        const int b = it & 1;
        const int tn = t + gridDim.x;
        // prefetch the next tile into the other buffer (freed at the end of
        // the previous iteration)
        if (tn < A.ntiles && threadIdx.x == 0 && staged(tn)) issue(tn, b ^ 1);
        const int bs = A.tile_brow[t], be = A.tile_brow[t + 1];
        const int j0 = A.rp[bs], j1 = A.rp[be];
        const bool use_smem = j1 - j0 <= A.cap_blocks && j1 > j0;
        if (use_smem) {
            const unsigned par = (b ? uses1 : uses0) & 1u;
            if (!mbar_wait_bounded(&bar[b], par)) {
                // record the phase that never completed; it is waited on
                // once more (bounded) before the CTA exits
                atomicOr(A.err, kErrTimeout);
                timed_out = 1 + (b << 1) + (par << 2);
            }
            if (b) ++uses1; else ++uses0;
        }
        const int nrows = (be - bs) * B;
        for (int lr = threadIdx.x; lr < nrows; lr += NT) {
            const int br = bs + lr / B, k = lr % B;
            const int jb = A.rp[br], je = A.rp[br + 1];
            float s = 0.f;
            // UJ blocks per round: their column indices and x segments are
            // all requested before the first product, so a block row costs
            // ceil(blocks / UJ) gather round trips instead of one per block.
            constexpr int UJ = B == 4 ? 8 : 4;
            for (int j = jb; j < je; j += UJ) {
                int cj[UJ];
#pragma unroll
                for (int u = 0; u < UJ; ++u) cj[u] = j + u < je ? __ldg(A.ci + j + u) : -1;
                float4 xv[UJ][B / 4];
#pragma unroll
                for (int u = 0; u < UJ; ++u)
#pragma unroll
                    for (int q = 0; q < B / 4; ++q)
                        xv[u][q] = cj[u] >= 0
                                       ? __ldg(reinterpret_cast<const float4*>(x + (size_t)cj[u] * B) + q)
                                       : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int u = 0; u < UJ; ++u) {
                    if (cj[u] < 0) break;
                    const float* row = use_smem ? buf[b] + (size_t)(j + u - j0) * BB + k * B
                                                : A.v + (size_t)(j + u) * BB + k * B;
                    const float4* r4 = reinterpret_cast<const float4*>(row);
                    float bsum = 0.f;
#pragma unroll
                    for (int q = 0; q < B / 4; ++q) {
                        const float4 a = r4[q];
                        bsum = fmaf(a.x, xv[u][q].x, bsum);
                        bsum = fmaf(a.y, xv[u][q].y, bsum);
                        bsum = fmaf(a.z, xv[u][q].z, bsum);
                        bsum = fmaf(a.w, xv[u][q].w, bsum);
                    }
                    s += bsum;
                }
            }
            epi.row(br * B + k, s, acc);
        }
        __syncthreads();   // buffer b may be refilled by the next iteration
    }
    // Drain: a prefetch is only issued for a tile this CTA processes and every
    // staged tile was waited on above, so a copy can only still be in flight
    // if its wait ran out; wait for that one again (bounded) before exiting.
    if (threadIdx.x == 0 && timed_out) {
        const int tb = (timed_out >> 1) & 1;
        const unsigned par = (unsigned)(timed_out >> 2) & 1u;
        mbar_wait_bounded(&bar[tb], par);
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

}  // namespace mps
