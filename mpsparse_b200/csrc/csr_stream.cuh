// csr_stream.cuh -- TMA-staged CSR SpMV for sm_100a (the hot kernel).
//
// Same tiles and epilogues as spmv_tiles (spmv_kernels.cuh), but the tile's
// col_ind, values and row_ptr segments are contiguous byte ranges, so one
// thread stages them into shared memory with bulk async copies
// (cp.async.bulk.shared::cluster.global, completion counted on an mbarrier; no
// multicast).  Two buffers per CTA: while the CTA multiplies tile t, the copy
// of its next tile is already in flight, so the HBM stream never waits for
// the per-tile reduction.  Per tile:
//   1. wait (bounded) for the tile's bytes;
//   2. one thread per nonzero: prod = val * x[col] (x gathered through the
//      read-only path and L2), written over the staged col_ind in place;
//   3. one thread (or warp, for long rows) per row sums its products using the
//      staged row_ptr and hands the sum to the epilogue.
// Tiles that do not fit a buffer (a row longer than the spare capacity, or
// more rows than the staged row_ptr holds) are reduced straight from global
// memory.  The handle's CSR arrays carry 16 spare elements so a copy rounded
// out to 16-byte boundaries never leaves its allocation.
#pragma once
#include "spmv_kernels.cuh"
#include "tma.cuh"

namespace mps {

template <bool BF16>
__host__ __device__ constexpr size_t stream_buf_bytes(int cap, int rcap) {
    return (size_t)cap * 4 + (size_t)cap * (BF16 ? 2 : 4) + (size_t)rcap * 4;
}

template <bool BF16, class Epi, int NT = kNT>
__global__ void __launch_bounds__(NT, 4)
spmv_stream(CsrStreamDev A, const float* __restrict__ x, Epi epi) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned long long bar[2];
    __shared__ double red[NT / 32];
    __shared__ float redf[NT / 32];
    __shared__ int last_flag;
    __shared__ int timed_out;
    if (blockIdx.x == 0 && threadIdx.x == 0) epi.tick();
    if (!epi.active()) {
        if (blockIdx.x == 0 && threadIdx.x == 0) epi.on_skip();
        return;
    }
    constexpr int GA = BF16 ? 8 : 4;   // elements per 16 bytes of the value array
    const size_t bb = stream_buf_bytes<BF16>(A.cap, A.rcap);
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

    auto staged = [&](const int4 m) {
        const int a0 = m.z & ~(GA - 1), a1 = (m.w + GA - 1) & ~(GA - 1);
        const int r0 = m.x & ~3, r1 = (m.y + 1 + 3) & ~3;
        return m.w > m.z && (a1 - a0) <= A.cap && (r1 - r0) <= A.rcap;
    };
    auto issue = [&](const int4 m, int b) {   // one thread
        const int a0 = m.z & ~(GA - 1), a1 = (m.w + GA - 1) & ~(GA - 1);
        const int r0 = m.x & ~3, r1 = (m.y + 1 + 3) & ~3;
        const unsigned bc = (unsigned)(a1 - a0) * 4u;
        const unsigned bv = (unsigned)(a1 - a0) * (BF16 ? 2u : 4u);
        const unsigned br = (unsigned)(r1 - r0) * 4u;
        unsigned char* base = smem + (size_t)b * bb;
        fence_proxy_async();
        mbar_expect_tx(&bar[b], bc + bv + br);
        bulk_g2s(base, A.ci + a0, bc, &bar[b]);
        if (BF16)
            bulk_g2s(base + (size_t)A.cap * 4, A.vb + a0, bv, &bar[b]);
        else
            bulk_g2s(base + (size_t)A.cap * 4, A.v + a0, bv, &bar[b]);
        bulk_g2s(base + (size_t)A.cap * (BF16 ? 6 : 8), A.rp + r0, br, &bar[b]);
    };

    unsigned uses0 = 0u, uses1 = 0u;   // completed phases per buffer (uniform)
    // Tile metadata: thread 0 keeps the next two tiles' {rs, re, k0, k1} in
    // registers (loaded two iterations ahead) and publishes the upcoming
    // tile's through shared memory, so no thread waits on a metadata load.
    __shared__ int4 s_meta[2];
    const int4 none = make_int4(0, 0, 0, 0);
    const int t0 = blockIdx.x, G = gridDim.x;
    int4 m_next = none, m_next2 = none;
    if (threadIdx.x == 0 && t0 < A.ntiles) {
        const int4 m0 = A.meta[t0];
        m_next = t0 + G < A.ntiles ? A.meta[t0 + G] : none;
        m_next2 = t0 + 2 * G < A.ntiles ? A.meta[t0 + 2 * G] : none;
        if (staged(m0)) issue(m0, 0);
        s_meta[0] = m0;
    }
    __syncthreads();
    int it = 0;
    for (int t = t0; t < A.ntiles; t += G, ++it) {
        const int b = it & 1;
        if (threadIdx.x == 0 && t + G < A.ntiles && staged(m_next)) issue(m_next, b ^ 1);
        const int4 m = s_meta[b];
        const int rs = m.x, re = m.y, k0 = m.z, k1 = m.w;
        if (rs < re) {
            if (staged(m)) {
                const unsigned par = (b ? uses1 : uses0) & 1u;
                if (!mbar_wait_bounded(&bar[b], par)) {
                    atomicOr(A.err, kErrTimeout);
                    timed_out = 1 + (b << 1) + (par << 2);
                }
                if (b) ++uses1; else ++uses0;
                unsigned char* base = smem + (size_t)b * bb;
                const int* cols = reinterpret_cast<const int*>(base);
                float* prod = reinterpret_cast<float*>(base);
                const int* rps = reinterpret_cast<const int*>(base + (size_t)A.cap * (BF16 ? 6 : 8));
                const int a0 = k0 & ~(GA - 1), r0 = rs & ~3;
                // products: U independent gathers in flight per thread (the
                // staged col_ind is overwritten by the products, so all loads
                // of a round are issued before any store)
                constexpr int U = 8;
                for (int kb = k0 + threadIdx.x; kb < k1; kb += NT * U) {
                    int c[U];
                    float v[U], xv[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int i = kb + u * NT - a0;
                        const bool in = kb + u * NT < k1;
                        c[u] = in ? cols[i] : -1;
                        if (BF16)
                            v[u] = in ? bf16_to_f(reinterpret_cast<const __nv_bfloat16*>(base + (size_t)A.cap * 4)[i]) : 0.f;
                        else
                            v[u] = in ? reinterpret_cast<const float*>(base + (size_t)A.cap * 4)[i] : 0.f;
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u) xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : 0.f;
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        if (kb + u * NT < k1) prod[kb + u * NT - a0] = v[u] * xv[u];
                }
                __syncthreads();
                const int nrows = re - rs;
                if ((k1 - k0) > 16 * nrows) {
                    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
                    for (int r = rs + wid; r < re; r += NT / 32) {
                        const int bgn = rps[r - r0] - a0, end = rps[r + 1 - r0] - a0;
                        float s = 0.f;
                        for (int k = bgn + lane; k < end; k += 32) s += prod[k];
                        s = warp_sum(s);
                        if (lane == 0) epi.row(r, s, acc);
                    }
                } else {
                    for (int r = rs + threadIdx.x; r < re; r += NT) {
                        const int bgn = rps[r - r0] - a0, end = rps[r + 1 - r0] - a0;
                        float s = 0.f;
                        for (int k = bgn; k < end; ++k) s += prod[k];
                        epi.row(r, s, acc);
                    }
                }
            } else {
                // not staged: short rows thread-per-row, long rows CTA-per-row
                for (int r = rs + threadIdx.x; r < re; r += NT) {
                    const int bgn = A.rp[r], end = A.rp[r + 1];
                    if (end - bgn <= 64) {
                        float s = 0.f;
                        for (int k = bgn; k < end; ++k) {
                            const float v = BF16 ? bf16_to_f(A.vb[k]) : ld_stream(A.v + k);
                            s += v * __ldg(x + ld_stream(A.ci + k));
                        }
                        epi.row(r, s, acc);
                    }
                }
                for (int r = rs; r < re; ++r) {
                    const int bgn = A.rp[r], end = A.rp[r + 1];
                    if (end - bgn <= 64) continue;
                    float s = 0.f;
                    for (int k = bgn + threadIdx.x; k < end; k += NT) {
                        const float v = BF16 ? bf16_to_f(A.vb[k]) : ld_stream(A.v + k);
                        s += v * __ldg(x + ld_stream(A.ci + k));
                    }
                    s = block_sum<NT>(s, redf);
                    if (threadIdx.x == 0) epi.row(r, s, acc);
                }
            }
        }
        if (threadIdx.x == 0) {
            s_meta[b ^ 1] = m_next;
            m_next = m_next2;
            m_next2 = t + 3 * G < A.ntiles ? A.meta[t + 3 * G] : none;
        }
        __syncthreads();   // buffer b is refilled by the next iteration's prefetch
    }
    if (threadIdx.x == 0 && timed_out) {   // a copy whose wait ran out: wait again, bounded
        mbar_wait_bounded(&bar[(timed_out >> 1) & 1], (unsigned)(timed_out >> 2) & 1u);
    }
    if constexpr (Epi::NS > 0) {
#pragma unroll
        for (int i = 0; i < Epi::NS; ++i) {
            const double v = block_sum<NT>(acc[i], red);
            if (threadIdx.x == 0) epi.partials[i * kMaxPartials + blockIdx.x] = v;
        }
        if (arrive_last(epi.counter, &last_flag)) {
            double tot[Epi::NS];
#pragma unroll
            for (int i = 0; i < Epi::NS; ++i)
                tot[i] = sum_partials<NT>(epi.partials + i * kMaxPartials, gridDim.x, red);
            if (threadIdx.x == 0) epi.finalize(tot);
        }
    }
}

}  // namespace mps
