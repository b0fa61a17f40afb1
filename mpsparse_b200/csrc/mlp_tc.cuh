// mlp_tc.cuh -- the learned-FSAI network (16 -> 64 -> 64 -> 1, GELU) on the
// 5th-generation tensor cores of sm_100a.
//
// Both kernels are persistent, 128 threads (4 warps) per CTA, 128 network rows
// (G nonzeros) per tile.  Operands live in shared memory in the canonical
// UMMA "no-swizzle" layouts (8-row x 16-byte core matrices); accumulators live
// in tensor memory (TMEM); one thread issues tcgen05.mma and tcgen05.commit
// signals an mbarrier; each warp reads its 32 TMEM lanes (= 32 rows) back with
// tcgen05.ld.32x32b.  BF16 operands, FP32 accumulation (kind::f16, A and B
// both BF16).
//
// Forward (per tile):  D1 = X W1  ->  h1 = GELU(D1 + b1) (BF16, to SMEM)
//                      D2 = h1 W2 ->  out = GELU(D2 + b2) . w3 + b3
// Backward (per tile, forward recomputed):
//   dz2 = dout * w3 * GELU'(z2)                     (BF16, to SMEM)
//   dh1 = dz2 W2^T                                  (MMA, K-major operands)
//   dW2 += [h1 | dz2]^T dz2   (MMA, M-major operands: the same SMEM tiles
//                              read transposed; rows 0..63 of the result)
//   dz1 = dh1 * GELU'(z1)                           (BF16, to SMEM)
//   dW1 += [x | 0 | dz1]^T dz1                      (rows 0..15)
// db1, db2, dw3, db3 are warp-shuffle reductions.  Weight-gradient
// accumulators stay in TMEM across a CTA's tiles and are added to global
// memory once at the end.  Every mbarrier wait is bounded; on a timeout the
// CTA records the error, waits once more (bounded) for its MMAs, frees its
// TMEM and returns.
#pragma once
#include "common.cuh"
#include "tma.cuh"

namespace mps {

constexpr int kNF = 16;
constexpr int kNH = 64;
constexpr int kNParam = kNF * kNH + kNH + kNH * kNH + kNH + kNH + 1;   // 5313
constexpr int kMlpRows = 128;
constexpr int kMlpThreads = 128;

// Packed weights (global memory, copied into SMEM by every CTA).
struct MlpPacked {
    __nv_bfloat16 w1t[kNH * kNF];   // B of D1: (n = out, k = in), canonical K-major
    __nv_bfloat16 w2t[kNH * kNH];   // B of D2: (n = out, k = in)
    __nv_bfloat16 w2[kNH * kNH];    // B of dh1: (n = in, k = out)
    float b1[kNH];
    float b2[kNH];
    float w3[kNH];                  // BF16-rounded values
    float b3;
    float pad_[3];
};

// Element offset of (row r, column k) in a canonical K-major no-swizzle tile
// with K columns: 8x8 core matrices (128 bytes), K-chunks of a row group
// adjacent, row groups after one another.
__host__ __device__ constexpr int canon(int r, int k, int K) {
    return ((r >> 3) * (K >> 3) + (k >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

// Shared-memory matrix descriptor (no swizzle): start, leading / stride byte
// offsets (16-byte units), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(const void* smem_ptr, unsigned lbo, unsigned sbo) {
    const unsigned a = smem_u32(smem_ptr);
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 A/B, FP32 D, M x N, majors.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) |
           ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         bool accumulate) {
    const uint32_t z = 0, acc = accumulate ? 1u : 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}
__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(unsigned* dst_smem, unsigned ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(dst_smem)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(unsigned taddr, unsigned ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}
// 32 lanes x 32 bit, 64 consecutive columns -> 64 registers of this lane.
__device__ __forceinline__ void tmem_ld64(unsigned taddr, float* v) {
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
        "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
        "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]),
          "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]),
          "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]),
          "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]),
          "=r"(r[62]), "=r"(r[63])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

// The network's activation: GELU in its tanh form (Hendrycks & Gimpel 2016),
//   gelu(x) = 0.5 x (1 + tanh(c (x + 0.044715 x^3))),  c = sqrt(2 / pi),
// with the SFU's tanh (tanh.approx.f32: about 11 correct bits, finer than the
// BF16 rounding of the activations that follows).  One SFU operation and a
// few FMAs per activation; the activations, not the MMAs, are the bulk of
// the network's instruction work (128 per row against 5 MMAs per 128 rows).
__device__ __forceinline__ float tanh_sfu(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kGeluC = 0.7978845608028654f;   // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;
__device__ __forceinline__ float gelu_f(float x) {
    const float t = tanh_sfu(kGeluC * fmaf(kGeluA * x, x * x, x));
    return 0.5f * x * (1.0f + t);
}
__device__ __forceinline__ float gelu_d(float x) {
    const float x2 = x * x;
    const float t = tanh_sfu(kGeluC * fmaf(kGeluA * x, x2, x));
    return fmaf(0.5f * x * kGeluC * fmaf(3.0f * kGeluA, x2, 1.0f), fmaf(-t, t, 1.0f), 0.5f * (1.0f + t));
}

// Eight FP32 values -> one 16-byte chunk of BF16 in SMEM.
__device__ __forceinline__ void store_bf16x8(__nv_bfloat16* dst, const float* v) {
    __nv_bfloat162 p[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(p);
}

// Copy the packed weights into SMEM (uint4 granules).
__device__ __forceinline__ void load_packed(const MlpPacked* __restrict__ g, MlpPacked* s) {
    const uint4* src = reinterpret_cast<const uint4*>(g);
    uint4* dst = reinterpret_cast<uint4*>(s);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 16); i += blockDim.x) dst[i] = src[i];
}

struct MlpFwdSmem {
    MlpPacked w;
    __nv_bfloat16 x[kMlpRows * kNF];   // canonical, K = 16
    __nv_bfloat16 h[kMlpRows * kNH];   // canonical, K = 64
    unsigned long long bar;
    unsigned taddr;
    int abort;
};
// Four forward CTAs per SM: 4 x 128 TMEM columns fill the SM's 512, and the
// launch asks for at least this much shared memory so that a fifth CTA never
// becomes resident (its TMEM allocation would wait for a column range).
constexpr int kMlpFwdCtasPerSm = 4;
constexpr size_t kMlpFwdSmemFloor = 50 * 1024;

// out[r] = net(X[r]) for r < N.  X is BF16 [N][16] (32 bytes per row).
__global__ void __launch_bounds__(kMlpThreads, kMlpFwdCtasPerSm)
mlp_forward_tc(const MlpPacked* __restrict__ wg, const __nv_bfloat16* __restrict__ X, long N,
               float* __restrict__ out, unsigned* err) {
    extern __shared__ __align__(1024) unsigned char mlp_smem[];
    MlpFwdSmem& S = *reinterpret_cast<MlpFwdSmem*>(mlp_smem);
    const int tid = threadIdx.x, warp = tid >> 5;
    load_packed(wg, &S.w);
    if (tid == 0) {
        mbar_init(&S.bar, 1);
        S.abort = 0;
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(&S.taddr, 128);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tbase = S.taddr;
    const unsigned lane_off = (unsigned)(warp * 32) << 16;
    const uint32_t idesc = umma_idesc(128, 64, false, false);
    unsigned phase = 0, pend_phase = 0;
    bool pending = false;
    const long ntiles = (N + kMlpRows - 1) / kMlpRows;
    for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long row = t * kMlpRows + tid;
        // X row -> SMEM (two 16-byte chunks)
        uint4 c0 = make_uint4(0, 0, 0, 0), c1 = c0;
        if (row < N) {
            const uint4* src = reinterpret_cast<const uint4*>(X + row * kNF);
            c0 = src[0];
            c1 = src[1];
        }
        *reinterpret_cast<uint4*>(S.x + canon(tid, 0, kNF)) = c0;
        *reinterpret_cast<uint4*>(S.x + canon(tid, 8, kNF)) = c1;
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            umma_f16(tbase, umma_desc(S.x, 128, 256), umma_desc(S.w.w1t, 128, 256), idesc, false);
            umma_commit(&S.bar);
        }
        if (!mbar_wait_bounded(&S.bar, phase)) {
            S.abort = 1;
            pending = true;
            pend_phase = phase;
        }
        phase ^= 1;
        tc_fence_after();
        float v[64];
        tmem_ld64(tbase + lane_off, v);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float hv[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) hv[i] = gelu_f(v[8 * c + i] + S.w.b1[8 * c + i]);
            store_bf16x8(S.h + canon(tid, 8 * c, kNH), hv);
        }
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        if (S.abort) break;
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int j = 0; j < 4; ++j)
                umma_f16(tbase + 64, umma_desc(S.h, 128, 1024) + (uint64_t)(16 * j),
                         umma_desc(S.w.w2t, 128, 1024) + (uint64_t)(16 * j), idesc, j > 0);
            umma_commit(&S.bar);
        }
        if (!mbar_wait_bounded(&S.bar, phase)) {
            S.abort = 1;
            pending = true;
            pend_phase = phase;
        }
        phase ^= 1;
        tc_fence_after();
        tmem_ld64(tbase + 64 + lane_off, v);
        float o = S.w.b3;
#pragma unroll
        for (int i = 0; i < 64; ++i) o = fmaf(gelu_f(v[i] + S.w.b2[i]), S.w.w3[i], o);
        if (row < N) out[row] = o;
        tc_fence_before();
        __syncthreads();
        if (S.abort) break;
    }
    if (S.abort) {
        if (tid == 0) atomicOr(err, kErrTimeout);
        if (pending) mbar_wait_bounded(&S.bar, pend_phase);   // the MMA that never signalled
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free(tbase, 128);
}

struct MlpBwdSmem {
    MlpPacked w;
    __nv_bfloat16 xd[kMlpRows * 128];   // [x (16) | 0 (48) | dz1 (64)], canonical K = 128
    __nv_bfloat16 hd[kMlpRows * 128];   // [h1 (64) | dz2 (64)],          canonical K = 128
    // per-warp sums over the CTA's rows (each lane owns two columns of its warp's row)
    float gb1[kMlpThreads / 32][kNH], gb2[kMlpThreads / 32][kNH], gw3[kMlpThreads / 32][kNH];
    float gb3[kMlpThreads / 32];
    unsigned long long bar;
    unsigned taddr;
    int abort;
};
// Two backward CTAs per SM: 2 x 256 TMEM columns; the shared memory of a CTA
// (about 85 KB) admits no third.
constexpr int kMlpBwdCtasPerSm = 2;

// Sum 64 per-row values over the warp's 32 rows by a butterfly
// reduce-scatter: in each of five rounds a lane keeps half of its values and
// sends the other half to its partner (32 + 16 + 8 + 4 + 2 independent
// shuffles in all, against 5 dependent ones for each of 64 separate
// reductions), ending with the totals of columns 2*lane and 2*lane + 1, which
// it adds to its warp's row of the accumulator (no atomics).  v is consumed.
template <int N>
__device__ __forceinline__ void rs_round(float* v, bool upper, int w) {
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
        const float keep = upper ? v[i + N / 2] : v[i];
        const float send = upper ? v[i] : v[i + N / 2];
        v[i] = keep + __shfl_xor_sync(kFull, send, w);
    }
}
__device__ __forceinline__ void warp_accum64(float* v, float* acc_row) {
    const int lane = threadIdx.x & 31;
    rs_round<64>(v, lane & 16, 16);
    rs_round<32>(v, lane & 8, 8);
    rs_round<16>(v, lane & 4, 4);
    rs_round<8>(v, lane & 2, 2);
    rs_round<4>(v, lane & 1, 1);
    acc_row[2 * lane] += v[0];
    acc_row[2 * lane + 1] += v[1];
}

// grad (FP32, parameter layout W1, b1, W2, b2, w3, b3) += d loss / d params
// for d loss / d out = dout.
__global__ void __launch_bounds__(kMlpThreads, kMlpBwdCtasPerSm)
mlp_backward_tc(const MlpPacked* __restrict__ wg, const __nv_bfloat16* __restrict__ X,
                const float* __restrict__ dout, long N, float* __restrict__ grad, unsigned* err) {
    extern __shared__ __align__(1024) unsigned char mlp_smem[];
    MlpBwdSmem& S = *reinterpret_cast<MlpBwdSmem*>(mlp_smem);
    const int tid = threadIdx.x, warp = tid >> 5;
    load_packed(wg, &S.w);
    for (int i = tid; i < (kMlpThreads / 32) * kNH; i += kMlpThreads)
        (&S.gb1[0][0])[i] = (&S.gb2[0][0])[i] = (&S.gw3[0][0])[i] = 0.f;
    if (tid < kMlpThreads / 32) S.gb3[tid] = 0.f;
    if (tid == 0) {
        mbar_init(&S.bar, 1);
        S.abort = 0;
        fence_mbar_init();
    }
    // zero feature columns 16..63 of xd (never written again)
    {
        const float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int c = 2; c < 8; ++c) store_bf16x8(S.xd + canon(tid, 8 * c, 128), z);
    }
    if (warp == 0) tmem_alloc(&S.taddr, 256);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tbase = S.taddr;
    const unsigned T_D1 = tbase, T_D2 = tbase + 64, T_W2 = tbase + 128, T_W1 = tbase + 192;
    const unsigned lane_off = (unsigned)(warp * 32) << 16;
    const uint32_t id_kk = umma_idesc(128, 64, false, false);
    const uint32_t id_mn = umma_idesc(128, 64, true, true);
    unsigned phase = 0;
    bool pending = false;
    int tiles_done = 0;
    const long ntiles = (N + kMlpRows - 1) / kMlpRows;
    unsigned pend_phase = 0;
    auto wait_mma = [&]() {
        if (!mbar_wait_bounded(&S.bar, phase)) {
            S.abort = 1;
            pending = true;
            pend_phase = phase;
        }
        phase ^= 1;
        tc_fence_after();
    };
    for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long row = t * kMlpRows + tid;
        const bool live = row < N;
        uint4 c0 = make_uint4(0, 0, 0, 0), c1 = c0;
        float d = 0.f;
        if (live) {
            const uint4* src = reinterpret_cast<const uint4*>(X + row * kNF);
            c0 = src[0];
            c1 = src[1];
            d = dout[row];
        }
        *reinterpret_cast<uint4*>(S.xd + canon(tid, 0, 128)) = c0;
        *reinterpret_cast<uint4*>(S.xd + canon(tid, 8, 128)) = c1;
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {                                   // D1 = X W1
            tc_fence_after();
            umma_f16(T_D1, umma_desc(S.xd, 128, 2048), umma_desc(S.w.w1t, 128, 256), id_kk, false);
            umma_commit(&S.bar);
        }
        wait_mma();
        float v[64];
        tmem_ld64(T_D1 + lane_off, v);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float hv[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) hv[i] = gelu_f(v[8 * c + i] + S.w.b1[8 * c + i]);
            store_bf16x8(S.hd + canon(tid, 8 * c, 128), hv);
        }
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        if (S.abort) break;
        if (tid == 0) {                                   // D2 = h1 W2
            tc_fence_after();
#pragma unroll
            for (int j = 0; j < 4; ++j)
                umma_f16(T_D2, umma_desc(S.hd, 128, 2048) + (uint64_t)(16 * j),
                         umma_desc(S.w.w2t, 128, 1024) + (uint64_t)(16 * j), id_kk, j > 0);
            umma_commit(&S.bar);
        }
        wait_mma();
        tmem_ld64(T_D2 + lane_off, v);
        {
            float h2[64];
#pragma unroll
            for (int i = 0; i < 64; ++i) {
                const float z = v[i] + S.w.b2[i];
                h2[i] = live ? d * gelu_f(z) : 0.f;              // dw3 contribution
                v[i] = live ? d * S.w.w3[i] * gelu_d(z) : 0.f;   // dz2
            }
#pragma unroll
            for (int c = 0; c < 8; ++c) store_bf16x8(S.hd + canon(tid, 64 + 8 * c, 128), v + 8 * c);
            warp_accum64(h2, S.gw3[warp]);
            warp_accum64(v, S.gb2[warp]);
            const float sd = warp_sum(d);
            if ((tid & 31) == 0) S.gb3[warp] += sd;
        }
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        if (S.abort) break;
        if (tid == 0) {
            tc_fence_after();
            // dh1 = dz2 W2^T  (D2's columns are free again)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                umma_f16(T_D2, umma_desc(S.hd + 64 * 8, 128, 2048) + (uint64_t)(16 * j),
                         umma_desc(S.w.w2, 128, 1024) + (uint64_t)(16 * j), id_kk, j > 0);
            // dW2 += [h1 | dz2]^T dz2, K = the 128 rows (8 steps of 16)
#pragma unroll
            for (int j = 0; j < 8; ++j)
                umma_f16(T_W2, umma_desc(S.hd, 2048, 128) + (uint64_t)(256 * j),
                         umma_desc(S.hd + 64 * 8, 2048, 128) + (uint64_t)(256 * j), id_mn,
                         tiles_done > 0 || j > 0);
            umma_commit(&S.bar);
        }
        wait_mma();
        float z1[64];
        tmem_ld64(T_D1 + lane_off, z1);
        tmem_ld64(T_D2 + lane_off, v);                    // dh1
#pragma unroll
        for (int i = 0; i < 64; ++i) v[i] = live ? v[i] * gelu_d(z1[i] + S.w.b1[i]) : 0.f;
#pragma unroll
        for (int c = 0; c < 8; ++c) store_bf16x8(S.xd + canon(tid, 64 + 8 * c, 128), v + 8 * c);
        warp_accum64(v, S.gb1[warp]);
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        if (S.abort) break;
        if (tid == 0) {                                   // dW1 += [x|0|dz1]^T dz1
            tc_fence_after();
#pragma unroll
            for (int j = 0; j < 8; ++j)
                umma_f16(T_W1, umma_desc(S.xd, 2048, 128) + (uint64_t)(256 * j),
                         umma_desc(S.xd + 64 * 8, 2048, 128) + (uint64_t)(256 * j), id_mn,
                         tiles_done > 0 || j > 0);
            umma_commit(&S.bar);
        }
        wait_mma();
        ++tiles_done;
        tc_fence_before();
        __syncthreads();
        if (S.abort) break;
    }
    if (S.abort) {
        if (tid == 0) atomicOr(err, kErrTimeout);
        if (pending) mbar_wait_bounded(&S.bar, pend_phase);   // the MMA that never signalled
    } else if (tiles_done > 0) {
        float* gW1 = grad;
        float* gb1 = gW1 + kNF * kNH;
        float* gW2 = gb1 + kNH;
        float* gb2 = gW2 + kNH * kNH;
        float* gw3 = gb2 + kNH;
        float* gb3 = gw3 + kNH;
        float v[64];
        if (warp < 2) {                                   // rows 0..63 of dW2's accumulator
            tmem_ld64(T_W2 + lane_off, v);
            const int f = tid;
            for (int o = 0; o < 64; ++o) atomicAdd(&gW2[f * kNH + o], v[o]);
        }
        if (warp == 0) {                                  // rows 0..15 of dW1's accumulator
            tmem_ld64(T_W1 + lane_off, v);
            if (tid < kNF)
                for (int o = 0; o < 64; ++o) atomicAdd(&gW1[tid * kNH + o], v[o]);
        }
        __syncthreads();
        for (int i = tid; i < kNH; i += kMlpThreads) {
            float a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
            for (int k = 0; k < kMlpThreads / 32; ++k) {
                a1 += S.gb1[k][i];
                a2 += S.gb2[k][i];
                a3 += S.gw3[k][i];
            }
            atomicAdd(&gb1[i], a1);
            atomicAdd(&gb2[i], a2);
            atomicAdd(&gw3[i], a3);
        }
        if (tid == 0) {
            float a = 0.f;
#pragma unroll
            for (int k = 0; k < kMlpThreads / 32; ++k) a += S.gb3[k];
            atomicAdd(gb3, a);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free(tbase, 256);
}

}  // namespace mps
