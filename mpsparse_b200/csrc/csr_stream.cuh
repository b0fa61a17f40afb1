// csr_stream.cuh -- TMA-staged CSR SpMV for sm_100a (the hot kernel).
//
// Same tiles and epilogues as spmv_tiles (spmv_kernels.cuh), but the tile's
// col_ind, values and row_ptr segments are contiguous byte ranges, so one
// thread stages them into shared memory with bulk async copies
// (cp.async.bulk.shared::cluster.global, completion counted on an mbarrier; no
// multicast) while the CTA multiplies earlier tiles.  Per tile:
//   1. wait (bounded) for the tile's bytes;
//   2. one thread per nonzero: prod = val * x[col] (x gathered through the
//      read-only path and L2), written over the staged col_ind in place;
//   3. one thread (or warp, for long rows) per row sums its products using the
//      staged row_ptr and hands the sum to the epilogue.
// Tiles that do not fit a buffer (a row longer than the spare capacity, or
// more rows than the staged row_ptr holds) are reduced straight from global
// memory.  The handle's CSR arrays carry 16 spare elements so a copy rounded
// out to 16-byte boundaries never leaves its allocation.
//
// Pipeline depth NB (buffers per CTA), chosen per matrix by the autotuner:
//   * NB == 2: the copy of tile it+1 is issued at the top of tile it, after
//     the barrier that ends tile it-1 (two block barriers per tile; the copy
//     overlaps all of tile it);
//   * NB >= 3: the copy of tile it+NB-1 is issued right after the barrier that
//     ends the product phase of tile it (by then every thread has finished
//     tile it-1, the buffer's last user), so each tile needs one barrier.
// col_ind/values are copied with an optional L2 evict-first policy so that x,
// gathered by every tile, stays resident in L2.
#pragma once
#include "spmv_kernels.cuh"
#include "tma.cuh"

namespace mps {

template <bool BF16>
__host__ __device__ constexpr size_t stream_buf_bytes(int cap, int rcap) {
    return (size_t)cap * 4 + (size_t)cap * (BF16 ? 2 : 4) + (size_t)rcap * 4;
}

// Two buffers leave room for 6 CTAs per SM (registers capped to match),
// three for 4: more warps in flight versus a deeper copy pipeline, chosen
// per matrix by the autotuner.  An epilogue that forms the multiplied vector
// on the fly keeps 4 CTAs per SM (64 registers): its gathers do not spill,
// and on a latency-bound 512^2 system 4 measured ~7% faster per iteration
// than 5 (fewer CTAs to launch, reduce and wait for).
template <class Epi, int NB>
constexpr int stream_min_ctas() {
    return NB == 2 ? (epi_has_gather<Epi>::value ? 4 : 6) : 4;
}

// Epilogues with `static constexpr bool kPre = true` run only inside solver
// loops, where the matrix does not change: the kernel requests its first
// tiles before waiting for the previous kernel of the stream (programmatic
// dependent launch), so the copies overlap that kernel's tail.
template <class E, class = void> struct epi_pre : std::false_type {};
template <class E> struct epi_pre<E, std::enable_if_t<E::kPre>> : std::true_type {};

template <bool BF16, class Epi, int NB, int NT = kNT>
__global__ void __launch_bounds__(NT, stream_min_ctas<Epi, NB>())
spmv_stream(CsrStreamDev A, const float* __restrict__ x, Epi epi) {
    static_assert(NB >= 2 && NB <= 4, "2 to 4 stages");
    constexpr bool PRE = epi_pre<Epi>::value;
    if constexpr (!PRE) pdl_begin();
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned long long bar[NB];
    __shared__ int4 s_meta[NB];
    __shared__ double red[(Epi::NS > 0 ? Epi::NS : 1) * (NT / 32)];
    __shared__ float redf[NT / 32];
    __shared__ int last_flag;
    __shared__ int timed_out;
    constexpr int GA = BF16 ? 8 : 4;   // elements per 16 bytes of the value array
    const size_t bb = stream_buf_bytes<BF16>(A.cap, A.rcap);

    auto staged = [&](const int4 m) {
        const int a0 = m.z & ~(GA - 1), a1 = (m.w + GA - 1) & ~(GA - 1);
        const int r0 = m.x & ~3, r1 = (m.y + 1 + 3) & ~3;
        return m.w > m.z && (a1 - a0) <= A.cap && (r1 - r0) <= A.rcap;
    };
    uint64_t pol = 0;
    const bool hint = A.evict_first != 0;
    auto issue = [&](const int4 m, int b) {   // one thread
        const int a0 = m.z & ~(GA - 1), a1 = (m.w + GA - 1) & ~(GA - 1);
        const int r0 = m.x & ~3, r1 = (m.y + 1 + 3) & ~3;
        const unsigned bc = (unsigned)(a1 - a0) * 4u;
        const unsigned bv = (unsigned)(a1 - a0) * (BF16 ? 2u : 4u);
        const unsigned br = (unsigned)(r1 - r0) * 4u;
        unsigned char* base = smem + (size_t)b * bb;
        fence_proxy_async();
        mbar_expect_tx(&bar[b], bc + bv + br);
        const void* vsrc = BF16 ? static_cast<const void*>(A.vb + a0) : static_cast<const void*>(A.v + a0);
        if (hint) {
            bulk_g2s_hint(base, A.ci + a0, bc, &bar[b], pol);
            bulk_g2s_hint(base + (size_t)A.cap * 4, vsrc, bv, &bar[b], pol);
        } else {
            bulk_g2s(base, A.ci + a0, bc, &bar[b]);
            bulk_g2s(base + (size_t)A.cap * 4, vsrc, bv, &bar[b]);
        }
        bulk_g2s(base + (size_t)A.cap * (BF16 ? 6 : 8), A.rp + r0, br, &bar[b]);
    };

    // Thread 0 loads the metadata of the next two tiles ahead into shared
    // memory (s_ahead, by cp.async: no registers held across the loop, no
    // wait on the load) and publishes each tile's through s_meta when it
    // issues the tile's copy.  At tile it, slot it & 1 holds tile
    // it + NB - 1 (issued next) and the other slot tile it + NB.
    __shared__ int4 s_ahead[2];
    const int4 none = make_int4(0, 0, 0, 0);
    const int t0 = blockIdx.x, G = gridDim.x;
    auto fetch_meta = [&](int ti, int slot) {   // thread 0
        if (ti < A.ntiles) cp_async16(&s_ahead[slot], A.meta + ti);
        else s_ahead[slot] = none;
    };
    unsigned issued = 0;           // thread 0: buffers the prologue filled
    auto prologue = [&]() {        // barriers and the first NB - 1 copies
        if (threadIdx.x != 0) return;
#pragma unroll
        for (int i = 0; i < NB; ++i) mbar_init(&bar[i], 1);
        timed_out = 0;
        fence_mbar_init();
        if (hint) pol = policy_evict_first();
        for (int i = 0; i < NB - 1; ++i) {
            const int ti = t0 + i * G;
            const int4 mi = ti < A.ntiles ? A.meta[ti] : none;
            if (ti < A.ntiles && staged(mi)) {
                issue(mi, i);
                issued |= 1u << i;
            }
            s_meta[i] = mi;
        }
        fetch_meta(t0 + (NB - 1) * G, 0);
        fetch_meta(t0 + NB * G, 1);
    };
    if constexpr (PRE) {
        prologue();
        pdl_begin();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) epi.tick();
    if (!epi.active()) {
        if (blockIdx.x == 0 && threadIdx.x == 0) epi.on_skip();
        if constexpr (PRE) {
            // the requested tiles land before the CTA (and its shared memory) goes
            if (threadIdx.x == 0)
                for (int i = 0; i < NB - 1; ++i)
                    if (((issued >> i) & 1u) && !mbar_wait_bounded(&bar[i], 0u)) atomicOr(A.err, kErrTimeout);
        }
        return;
    }
    epi_begin(epi);
    if constexpr (!PRE) prologue();
    double acc[Epi::NS > 0 ? Epi::NS : 1];
#pragma unroll
    for (int i = 0; i < (Epi::NS > 0 ? Epi::NS : 1); ++i) acc[i] = 0.0;
    __syncthreads();
    // Issue the copy of tile it + NB - 1 into the buffer tile it - 1 used.
    auto issue_ahead = [&](int t, int it) {   // one thread
        const int bn = (it + NB - 1) % NB;
        cp_async_wait_all();
        const int4 ma = s_ahead[it & 1];
        if (t + (NB - 1) * G < A.ntiles && staged(ma)) issue(ma, bn);
        s_meta[bn] = ma;
        fetch_meta(t + (NB + 1) * G, it & 1);
    };
    unsigned phase_bits = 0u;      // completed-phase parity per buffer (uniform)
    int it = 0;
    for (int t = t0; t < A.ntiles; t += G, ++it) {
        const int b = it % NB;
        if constexpr (NB == 2) {
            if (it > 0) __syncthreads();      // every thread is done with tile it - 1
            if (threadIdx.x == 0) issue_ahead(t, it);
        }
        const int4 m = s_meta[b];
        const int rs = m.x, re = m.y, k0 = m.z, k1 = m.w;
        const bool stg = rs < re && staged(m);
        // long rows (over 16 nonzeros on average): products first, then one
        // warp per row; short rows: one thread per row forms and adds its own
        // products (same products, same order), with no product phase and no
        // barrier between the phases
        const bool two_phase = stg && (k1 - k0) > 16 * (re - rs);
        unsigned char* base = smem + (size_t)b * bb;
        const int a0 = k0 & ~(GA - 1), r0 = rs & ~3;
        if (stg) {
            const unsigned par = (phase_bits >> b) & 1u;
            if (!mbar_wait_bounded(&bar[b], par)) {
                atomicOr(A.err, kErrTimeout);
                timed_out = 1 + (b << 1) + (par << 3);
            }
            phase_bits ^= 1u << b;
        }
        if (two_phase) {
            const int* cols = reinterpret_cast<const int*>(base);
            float* prod = reinterpret_cast<float*>(base);
            // products: U independent gathers in flight per thread (the staged
            // col_ind is overwritten by the products, so all loads of a round
            // are issued before any store)
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
                for (int u = 0; u < U; ++u) xv[u] = c[u] >= 0 ? epi_x(epi, x, c[u]) : 0.f;
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (kb + u * NT < k1) prod[kb + u * NT - a0] = v[u] * xv[u];
            }
        }
        // Products visible (two-phase tiles).  With NB >= 3, every thread is
        // past tile it - 1, so its buffer takes the copy of tile it + NB - 1.
        if (NB >= 3 || two_phase) __syncthreads();
        if constexpr (NB >= 3) {
            if (threadIdx.x == 0) issue_ahead(t, it);
        }
        if (rs < re) {
            if (stg) {
                const int* rps = reinterpret_cast<const int*>(base + (size_t)A.cap * (BF16 ? 6 : 8));
                if (two_phase) {
                    const float* prod = reinterpret_cast<const float*>(base);
                    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
                    for (int r = rs + wid; r < re; r += NT / 32) {
                        const int bgn = rps[r - r0] - a0, end = rps[r + 1 - r0] - a0;
                        float s = 0.f;
                        for (int k = bgn + lane; k < end; k += 32) s += prod[k];
                        s = warp_sum(s);
                        if (lane == 0) epi.row(r, s, acc);
                    }
                } else {
                    // rows r and r + NT together: the gathers of both rows are
                    // issued four at a time before their products are added,
                    // so a thread's two rows cost one gather round trip (only
                    // the gathered values stay live; the matrix values are
                    // read from shared memory as they are multiplied)
                    const int* cols = reinterpret_cast<const int*>(base);
                    const unsigned char* vbase = base + (size_t)A.cap * 4;
                    auto val = [&](int i) {
                        if constexpr (BF16) return bf16_to_f(reinterpret_cast<const __nv_bfloat16*>(vbase)[i]);
                        else return reinterpret_cast<const float*>(vbase)[i];
                    };
                    for (int r = rs + threadIdx.x; r < re; r += 2 * NT) {
                        const int r2 = r + NT;
                        const bool has2 = r2 < re;
                        const int b1 = rps[r - r0] - a0, e1 = rps[r + 1 - r0] - a0;
                        const int b2 = has2 ? rps[r2 - r0] - a0 : 0, e2 = has2 ? rps[r2 + 1 - r0] - a0 : 0;
                        float s1 = 0.f, s2 = 0.f;
                        const int len = max(e1 - b1, e2 - b2);
                        for (int k = 0; k < len; k += 4) {
                            float g1[4], g2[4];
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                g1[u] = b1 + k + u < e1 ? epi_x(epi, x, cols[b1 + k + u]) : 0.f;
                                g2[u] = b2 + k + u < e2 ? epi_x(epi, x, cols[b2 + k + u]) : 0.f;
                            }
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                if (b1 + k + u < e1) s1 = __fadd_rn(s1, __fmul_rn(val(b1 + k + u), g1[u]));
                                if (b2 + k + u < e2) s2 = __fadd_rn(s2, __fmul_rn(val(b2 + k + u), g2[u]));
                            }
                        }
                        epi.row(r, s1, acc);
                        if (has2) epi.row(r2, s2, acc);
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
                            s += v * epi_x(epi, x, ld_stream(A.ci + k));
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
                        s += v * epi_x(epi, x, ld_stream(A.ci + k));
                    }
                    s = block_sum<NT>(s, redf);
                    if (threadIdx.x == 0) epi.row(r, s, acc);
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && timed_out) {   // a copy whose wait ran out: wait again, bounded
        mbar_wait_bounded(&bar[(timed_out >> 1) & 3], (unsigned)(timed_out >> 3) & 1u);
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
