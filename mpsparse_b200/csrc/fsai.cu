// fsai.cu -- learned factorized sparse approximate inverse (FSAI) preconditioner.
//
// G is lower triangular on the pattern of tril(A); PCG applies M^-1 = G^T G
// (z = G^T (G r)), which is SPD whenever G's diagonal is positive.  Every
// nonzero (i, j) of G gets 16 features from A's local coefficients; the
// network (mlp_tc.cuh, tensor cores) maps them to o_ij and
//     g_ii = softplus(o_ii + c) / sqrt(a_ii),  g_ij = o_ij / sqrt(a_jj),
// c = log(e - 1), so G is nonsingular by construction and a network that
// outputs zero gives G = D^-1/2 (Jacobi).  Training minimises the probe estimate
// L = sum_v ||v - G A G^T v||^2 / (k n) of ||I - G A G^T||_F^2 / n with
// Rademacher probes plus caller-supplied vectors (e.g. CG residuals of the
// system), using
//     dL/dg_ij = 2/(k n) sum_v (e_i w_j + v_i s_j),
//     w = A G^T v, e = G w - v, s = A G^T e,
// then the network's backward pass and Adam.  No reference counterpart.
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "handles.hpp"
#include "mlp_tc.cuh"

namespace mps {
namespace {

// Per-row inputs of the features: float4 {diag, dd, near-lower coef, far-lower
// coef}, float4 {near-upper coef, far-upper coef, 0, 0}, int4 {near-lower col,
// far-lower col, near-upper col, far-upper col} (-1: none).
struct RowInfoDev {
    float4* f0;
    float4* f1;
    int4* c;
};

__global__ void g_count_kernel(const int* __restrict__ rp, const int* __restrict__ ci, int n,
                               unsigned* __restrict__ cnt) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        unsigned c = 0;
        for (int k = rp[r]; k < rp[r + 1]; ++k) c += ci[k] <= r;
        cnt[r] = c;
    }
}

__global__ void g_fill_kernel(const int* __restrict__ rp, const int* __restrict__ ci, int n,
                              const int* __restrict__ g_rp, int* __restrict__ g_ci,
                              int* __restrict__ g_row, int* __restrict__ g_aidx) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        int o = g_rp[r];
        for (int k = rp[r]; k < rp[r + 1]; ++k)
            if (ci[k] <= r) {
                g_ci[o] = ci[k];
                g_row[o] = r;
                g_aidx[o] = k;
                ++o;
            }
    }
}

__global__ void row_info_kernel(const int* __restrict__ rp, const int* __restrict__ ci,
                                const float* __restrict__ v, int n, RowInfoDev ri) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        float diag = 0.f, off = 0.f, lnv = 0.f, lfv = 0.f, unv = 0.f, ufv = 0.f;
        int ln = -1, lf = -1, un = -1, uf = -1;
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            const int c = ci[k];
            const float a = v[k];
            if (c == r) {
                diag += a;
                continue;
            }
            off += fabsf(a);
            if (c < r) {
                lf = ln;
                lfv = lnv;
                ln = c;
                lnv = a;
            } else if (un < 0) {
                un = c;
                unv = a;
            } else if (uf < 0) {
                uf = c;
                ufv = a;
            }
        }
        const float dd = diag != 0.f ? (diag - off) / diag : 0.f;
        ri.f0[r] = make_float4(diag, dd, lnv, lfv);
        ri.f1[r] = make_float4(unv, ufv, 0.f, 0.f);
        ri.c[r] = make_int4(ln, lf, un, uf);
    }
}

__device__ __forceinline__ float nrm(float a, float di, float dj) { return a / sqrtf(di * dj); }

// The 16 features of G nonzero k = (i, j) (see orc_fsai_features).
__global__ void features_kernel(long nnz_g, const int* __restrict__ g_row, const int* __restrict__ g_ci,
                                const int* __restrict__ g_aidx, const float* __restrict__ av,
                                RowInfoDev ri, __nv_bfloat16* __restrict__ X, float* __restrict__ Xf) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nnz_g;
         k += (long)gridDim.x * blockDim.x) {
        const int i = g_row[k], j = g_ci[k];
        const float4 a0 = ri.f0[i], a1 = ri.f1[i], b0 = ri.f0[j];
        const int4 ca = ri.c[i], cb = ri.c[j];
        const float di = a0.x, dj = b0.x;
        float f[16];
        f[0] = 1.f;
        f[1] = i == j ? 1.f : 0.f;
        f[2] = j == ca.x ? 1.f : 0.f;
        f[3] = j == ca.y ? 1.f : 0.f;
        f[4] = ca.x >= 0 ? nrm(a0.z, di, ri.f0[ca.x].x) : 0.f;
        f[5] = ca.y >= 0 ? nrm(a0.w, di, ri.f0[ca.y].x) : 0.f;
        f[6] = ca.z >= 0 ? nrm(a1.x, di, ri.f0[ca.z].x) : 0.f;
        f[7] = ca.w >= 0 ? nrm(a1.y, di, ri.f0[ca.w].x) : 0.f;
        f[8] = ca.x >= 0 ? logf(di / ri.f0[ca.x].x) : 0.f;
        f[9] = ca.y >= 0 ? logf(di / ri.f0[ca.y].x) : 0.f;
        f[10] = i == j ? 1.f : nrm(av[g_aidx[k]], di, dj);
        f[11] = logf(di / dj);
        f[12] = a0.y;
        f[13] = b0.y;
        f[14] = cb.x >= 0 ? nrm(b0.z, dj, ri.f0[cb.x].x) : 0.f;
        f[15] = cb.y >= 0 ? nrm(b0.w, dj, ri.f0[cb.y].x) : 0.f;
        __nv_bfloat162 p[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) p[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
        uint4* dst = reinterpret_cast<uint4*>(X + k * kNF);
        dst[0] = *reinterpret_cast<const uint4*>(&p[0]);
        dst[1] = *reinterpret_cast<const uint4*>(&p[4]);
        if (Xf)
#pragma unroll
            for (int q = 0; q < 16; ++q) Xf[k * kNF + q] = f[q];
    }
}

// Network output -> G values, and d g / d out.
__global__ void gvals_kernel(long nnz_g, const int* __restrict__ g_row, const int* __restrict__ g_ci,
                             const float* __restrict__ out, RowInfoDev ri, float* __restrict__ gv,
                             float* __restrict__ dgdo) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nnz_g;
         k += (long)gridDim.x * blockDim.x) {
        const int i = g_row[k], j = g_ci[k];
        const float o = out[k];
        const float s = rsqrtf(ri.f0[j].x);
        if (i == j) {
            const float z = o + 0.54132485f;                     // softplus(c) = 1
            const float sp = z > 20.f ? z : log1pf(expf(z));
            gv[k] = sp * s;
            dgdo[k] = s / (1.f + expf(-z));
        } else {
            gv[k] = o * s;
            dgdo[k] = s;
        }
    }
}

__global__ void gather_kernel(long n, const uint32_t* __restrict__ perm, const float* __restrict__ src,
                              float* __restrict__ dst) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        dst[k] = src[perm[k]];
}

__device__ __forceinline__ uint32_t mix32(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return (uint32_t)x;
}

__global__ void rademacher_kernel(int n, uint64_t seed, float* __restrict__ v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v[i] = (mix32(seed * 0x9E3779B97F4A7C15ull + (uint64_t)i) & 1u) ? 1.f : -1.f;
}

// y = G w -> e = y - v ; ||e||^2 accumulated into *loss
struct EpiProbeE {
    static constexpr int NS = 1;
    float* e;
    const float* v;
    double* loss;
    unsigned* counter;
    double* partials;
    __device__ void tick() const {}
    __device__ bool active() const { return true; }
    __device__ void on_skip() const {}
    __device__ void row(int r, float s, double* acc) const {
        const float d = s - v[r];
        e[r] = d;
        acc[0] += (double)d * (double)d;
    }
    __device__ void finalize(const double* tot) const { *loss += tot[0]; }
};

__global__ void grad_accum_kernel(long nnz_g, const int* __restrict__ g_row, const int* __restrict__ g_ci,
                                  const float* __restrict__ e, const float* __restrict__ w,
                                  const float* __restrict__ v, const float* __restrict__ s,
                                  float* __restrict__ grad) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nnz_g;
         k += (long)gridDim.x * blockDim.x) {
        const int i = g_row[k], j = g_ci[k];
        grad[k] += e[i] * w[j] + v[i] * s[j];
    }
}

__global__ void scale_kernel(long n, float* __restrict__ a, const float* __restrict__ b, float sc) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        a[k] = b ? a[k] * b[k] * sc : a[k] * sc;
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float c1, float c2) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = isfinite(g[i]) ? g[i] : 0.f;
        m[i] = b1 * m[i] + (1.f - b1) * gi;
        v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
        p[i] -= lr * (m[i] * c1) / (sqrtf(v[i] * c2) + eps);
    }
}

// FP32 parameters -> packed BF16 canonical operands + FP32 vectors.
__global__ void pack_kernel(const float* __restrict__ p, MlpPacked* __restrict__ w) {
    const float* W1 = p;
    const float* b1 = W1 + kNF * kNH;
    const float* W2 = b1 + kNH;
    const float* b2 = W2 + kNH * kNH;
    const float* w3 = b2 + kNH;
    const float* b3 = w3 + kNH;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < kNH * kNH; t += gridDim.x * blockDim.x) {
        const int a = t / kNH, b = t % kNH;
        // w2t: (n = out b? ) -- element (n, k) = W2[k][n]
        w->w2t[canon(a, b, kNH)] = __float2bfloat16_rn(W2[b * kNH + a]);   // n = a (out), k = b (in)
        w->w2[canon(a, b, kNH)] = __float2bfloat16_rn(W2[a * kNH + b]);    // n = a (in),  k = b (out)
        if (t < kNH * kNF) {
            const int n = t / kNF, k = t % kNF;                            // n = out, k = in
            w->w1t[canon(n, k, kNF)] = __float2bfloat16_rn(W1[k * kNH + n]);
        }
        if (t < kNH) {
            w->b1[t] = b1[t];
            w->b2[t] = b2[t];
            w->w3[t] = __bfloat162float(__float2bfloat16_rn(w3[t]));
        }
        if (t == 0) {
            w->b3 = b3[0];
            w->pad_[0] = w->pad_[1] = w->pad_[2] = 0.f;
        }
    }
}

int g1(long n) {
    long g = (n + 255) / 256, c = (long)num_sms() * 8;
    return (int)(g < 1 ? 1 : (g > c ? c : g));
}

}  // namespace

void fsai_work_free(FsaiWork& w) {
    dev_free(w.g_row);
    dev_free(w.g_aidx);
    dev_free(w.perm);
    dev_free(w.X);
    dev_free(w.out);
    dev_free(w.dgdo);
    dev_free(w.grad);
    dev_free(w.rinfo);
    dev_free(w.d_loss);
    dev_free(w.vec);
    w = FsaiWork{};
}

static RowInfoDev rinfo_of(const FsaiWork& w, int n) {
    float4* f = reinterpret_cast<float4*>(w.rinfo);
    return RowInfoDev{f, f + n, reinterpret_cast<int4*>(f + 2 * (size_t)n)};
}

// idx[k] = k: the payload that turns the sorted G^T keys into the permutation.
static __global__ void iota_kernel(uint32_t* __restrict__ idx, long n) {
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
        idx[k] = (uint32_t)k;
}

// G's pattern, G^T (pattern + permutation), per-row info and the features.
static mps_status fsai_prepare(mps_csr* h, cudaStream_t s) {
    FsaiWork& w = h->fw;
    if (w.ready) return MPS_OK;
    const CsrMat& A = h->A;
    const int n = (int)A.n_rows;
    if (A.n_rows != A.n_cols) return fail(MPS_ERR_ARG, "FSAI needs a square matrix");
    unsigned* cnt = nullptr;
    unsigned* bsum = nullptr;
    MPS_CUDA(stream_alloc(&cnt, ((size_t)n + 1) * 4, s));
    MPS_CUDA(stream_alloc(&bsum, (((size_t)n + 2048) / 2048 + 1) * 4, s));
    g_count_kernel<<<g1(n), 256, 0, s>>>(A.rp, A.ci, n, cnt);
    fsai_product_free(h);
    csr_free(h->G);
    csr_free(h->Gt);
    h->has_fsai = false;
    h->H.drop_graphs();
    // the pattern size is needed on the host for the allocations
    int32_t* grp_tmp = nullptr;
    MPS_CUDA(stream_alloc(&grp_tmp, ((size_t)n + 1) * 4, s));
    MPS_CUDA(exclusive_scan_rows(cnt, n, grp_tmp, bsum, s));
    int nnz_g = 0;
    MPS_CUDA(cudaMemcpyAsync(&nnz_g, grp_tmp + n, 4, cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaStreamSynchronize(s));
    mps_status st = alloc_csr(h->G, n, n, (uint64_t)nnz_g, h->d_err, s);
    if (st != MPS_OK) return st;
    MPS_CUDA(cudaMemcpyAsync(h->G.rp, grp_tmp, ((size_t)n + 1) * 4, cudaMemcpyDeviceToDevice, s));
    const size_t nz = (size_t)nnz_g + kCsrPad;
    MPS_CUDA(dev_alloc(&w.g_row, nz * 4, s));
    MPS_CUDA(dev_alloc(&w.g_aidx, nz * 4, s));
    MPS_CUDA(dev_alloc(&w.perm, nz * 4, s));
    MPS_CUDA(dev_alloc(&w.X, nz * kNF * 2, s));
    MPS_CUDA(dev_alloc(&w.out, nz * 4, s));
    MPS_CUDA(dev_alloc(&w.dgdo, nz * 4, s));
    MPS_CUDA(dev_alloc(&w.grad, nz * 4, s));
    MPS_CUDA(dev_alloc(&w.rinfo, (size_t)n * 48, s));
    MPS_CUDA(dev_alloc(&w.d_loss, 8, s));
    MPS_CUDA(dev_alloc(&w.vec, 6 * ((size_t)n + 4) * 4, s));
    g_fill_kernel<<<g1(n), 256, 0, s>>>(A.rp, A.ci, n, h->G.rp, h->G.ci, w.g_row, w.g_aidx);
    // (G's SpMV plan is built below, with G^T's, by factor_plans_follow)
    // G^T: sort (col << 32 | row) keys with the G index as payload
    unsigned long long* keys = nullptr;
    uint32_t* idx = nullptr;
    MPS_CUDA(stream_alloc(&keys, nz * 8, s));
    MPS_CUDA(stream_alloc(&idx, nz * 4, s));
    MPS_CUDA(transpose_keys_launch(h->G, keys, s));
    iota_kernel<<<g1(nnz_g), 256, 0, s>>>(idx, (long)nnz_g);
    MPS_CUDA(cudaGetLastError());
    st = build_from_keys(h->Gt, reinterpret_cast<const uint64_t*>(keys), idx, (uint64_t)nnz_g, n, n,
                         h->d_err, s, false);   // plans: factor_plans_follow below
    cudaFreeAsync(keys, s);
    cudaFreeAsync(idx, s);
    if (st != MPS_OK) return st;
    // the sorted payload landed in Gt.v: it is the permutation
    MPS_CUDA(cudaMemcpyAsync(w.perm, h->Gt.v, (size_t)nnz_g * 4, cudaMemcpyDeviceToDevice, s));
    MPS_CUDA(factor_plans_follow(h, s));
    RowInfoDev ri = rinfo_of(w, n);
    row_info_kernel<<<g1(n), 256, 0, s>>>(A.rp, A.ci, A.v, n, ri);
    features_kernel<<<g1(nnz_g), 256, 0, s>>>(nnz_g, w.g_row, h->G.ci, w.g_aidx, A.v, ri, w.X, nullptr);
    MPS_CUDA(cudaGetLastError());
    cudaFreeAsync(cnt, s);
    cudaFreeAsync(bsum, s);
    cudaFreeAsync(grp_tmp, s);
    w.nnz_g = (uint64_t)nnz_g;
    w.ready = true;
    return MPS_OK;
}

static cudaError_t mlp_forward_launch(const MlpPacked* wp, const __nv_bfloat16* X, long N, float* out,
                                      unsigned* err, cudaStream_t s) {
    const size_t smem = sizeof(MlpFwdSmem) > kMlpFwdSmemFloor ? sizeof(MlpFwdSmem) : kMlpFwdSmemFloor;
    static_assert(sizeof(MlpFwdSmem) + 1024 <= (228 * 1024) / kMlpFwdCtasPerSm, "forward CTAs per SM");
    static_assert((kMlpFwdSmemFloor + 1024) * (kMlpFwdCtasPerSm + 1) > 228 * 1024, "at most 4 per SM");
    cudaFuncSetAttribute(mlp_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    long tiles = (N + kMlpRows - 1) / kMlpRows;
    int grid = num_sms() * kMlpFwdCtasPerSm;
    if (tiles < grid) grid = (int)(tiles > 0 ? tiles : 1);
    mlp_forward_tc<<<grid, kMlpThreads, smem, s>>>(wp, X, N, out, err);
    return cudaGetLastError();
}

static cudaError_t mlp_backward_launch(const MlpPacked* wp, const __nv_bfloat16* X, const float* dout,
                                       long N, float* grad, unsigned* err, cudaStream_t s) {
    const size_t smem = sizeof(MlpBwdSmem);
    static_assert(sizeof(MlpBwdSmem) + 1024 <= (228 * 1024) / kMlpBwdCtasPerSm, "backward CTAs per SM");
    static_assert((sizeof(MlpBwdSmem) + 1024) * (kMlpBwdCtasPerSm + 1) > 228 * 1024, "at most 2 per SM");
    cudaFuncSetAttribute(mlp_backward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    long tiles = (N + kMlpRows - 1) / kMlpRows;
    int grid = num_sms() * kMlpBwdCtasPerSm;
    if (tiles < grid) grid = (int)(tiles > 0 ? tiles : 1);
    mlp_backward_tc<<<grid, kMlpThreads, smem, s>>>(wp, X, dout, N, grad, err);
    return cudaGetLastError();
}

}  // namespace mps

using namespace mps;

struct mps_fsai_model {
    float* params = nullptr;   // FP32 master weights
    float* m = nullptr;        // Adam moments
    float* v = nullptr;
    float* grad = nullptr;
    MlpPacked* packed = nullptr;
    unsigned* err = nullptr;
    int step = 0;
};

// Network output -> G values on h's pattern; G^T values by permutation.
static mps_status fsai_values(mps_csr* h, const mps_fsai_model* m, cudaStream_t s) {
    FsaiWork& w = h->fw;
    const long nz = (long)w.nnz_g;
    MPS_CUDA(mlp_forward_launch(m->packed, w.X, nz, w.out, m->err, s));
    gvals_kernel<<<g1(nz), 256, 0, s>>>(nz, w.g_row, h->G.ci, w.out, rinfo_of(w, (int)h->A.n_rows),
                                        h->G.v, w.dgdo);
    gather_kernel<<<g1(nz), 256, 0, s>>>(nz, w.perm, h->G.v, h->Gt.v);
    MPS_CUDA(cudaGetLastError());
    return MPS_OK;
}

static __global__ void fold_error_kernel(const unsigned* __restrict__ src, unsigned* dst) {
    const unsigned e = *src;
    if (e) atomicOr(dst, e);
}

static mps_status model_error(const mps_fsai_model* m, cudaStream_t s) {
    unsigned e = 0;
    MPS_CUDA(cudaMemcpyAsync(&e, m->err, 4, cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaStreamSynchronize(s));
    if (e & kErrTimeout) return fail(MPS_ERR_TIMEOUT, "FSAI network: a tensor-core wait gave up");
    return MPS_OK;
}

extern "C" {

int32_t mps_fsai_param_count(void) { return kNParam; }

mps_status mps_fsai_model_create(const float* h_params, mps_fsai_model** out) {
    if (!out) return fail(MPS_ERR_ARG, "out is null");
    *out = nullptr;
    mps_fsai_model* m = new mps_fsai_model();
    std::vector<float> p(kNParam, 0.f);
    if (h_params) {
        std::memcpy(p.data(), h_params, kNParam * sizeof(float));
    } else {
        // deterministic start: small random weights and a near-zero output,
        // so the untrained factor is close to Jacobi (G = D^-1/2)
        std::mt19937 rng(12345);
        std::normal_distribution<float> nd(0.f, 1.f);
        for (int i = 0; i < kNF * kNH; ++i) p[i] = nd(rng) * 0.25f;
        float* W2 = p.data() + kNF * kNH + kNH;
        for (int i = 0; i < kNH * kNH; ++i) W2[i] = nd(rng) * 0.125f;
        float* w3 = W2 + kNH * kNH + kNH;
        for (int i = 0; i < kNH; ++i) w3[i] = nd(rng) * 0.01f;
    }
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc(&m->params, kNParam * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->m, kNParam * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->v, kNParam * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->grad, kNParam * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->packed, sizeof(MlpPacked));
    if (e == cudaSuccess) e = cudaMalloc(&m->err, 4);
    if (e == cudaSuccess) e = cudaMemcpy(m->params, p.data(), kNParam * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->m, 0, kNParam * 4);
    if (e == cudaSuccess) e = cudaMemset(m->v, 0, kNParam * 4);
    if (e == cudaSuccess) e = cudaMemset(m->err, 0, 4);
    if (e == cudaSuccess) {
        pack_kernel<<<16, 256>>>(m->params, m->packed);
        e = cudaDeviceSynchronize();
    }
    if (e != cudaSuccess) {
        mps_fsai_model_destroy(m);
        return cuda_fail(e, "fsai_model_create");
    }
    *out = m;
    return MPS_OK;
}

mps_status mps_fsai_model_destroy(mps_fsai_model* m) {
    if (!m) return MPS_OK;
    cudaFree(m->params);
    cudaFree(m->m);
    cudaFree(m->v);
    cudaFree(m->grad);
    cudaFree(m->packed);
    cudaFree(m->err);
    delete m;
    return MPS_OK;
}

mps_status mps_fsai_model_get(const mps_fsai_model* m, float* h_params) {
    if (!m || !h_params) return fail(MPS_ERR_ARG, "null argument");
    MPS_CUDA(cudaMemcpy(h_params, m->params, kNParam * 4, cudaMemcpyDeviceToHost));
    return MPS_OK;
}

mps_status mps_fsai_model_set(mps_fsai_model* m, const float* h_params) {
    if (!m || !h_params) return fail(MPS_ERR_ARG, "null argument");
    MPS_CUDA(cudaMemcpy(m->params, h_params, kNParam * 4, cudaMemcpyHostToDevice));
    MPS_CUDA(cudaMemset(m->m, 0, kNParam * 4));
    MPS_CUDA(cudaMemset(m->v, 0, kNParam * 4));
    m->step = 0;
    pack_kernel<<<16, 256>>>(m->params, m->packed);
    MPS_CUDA(cudaDeviceSynchronize());
    return MPS_OK;
}

mps_status mps_fsai_attach(mps_csr* h, const mps_fsai_model* m, cudaStream_t s) {
    if (!h || !m) return fail(MPS_ERR_ARG, "null argument");
    mps_status st = fsai_prepare(h, s);
    if (st != MPS_OK) return st;
    st = fsai_values(h, m, s);
    if (st != MPS_OK) return st;
    // no synchronisation: the network's error word is folded into the
    // handle's second error word and reported by the next solve
    fold_error_kernel<<<1, 1, 0, s>>>(m->err, h->d_err + 1);
    MPS_CUDA(cudaGetLastError());
    h->has_fsai = true;
    return fsai_factor_changed(h, s);
}

mps_status mps_fsai_features(mps_csr* h, float* d_X, int32_t* d_g_row_ptr, int32_t* d_g_col_ind,
                             uint64_t* nnz_g, cudaStream_t s) {
    if (!h) return fail(MPS_ERR_ARG, "null handle");
    mps_status st = fsai_prepare(h, s);
    if (st != MPS_OK) return st;
    FsaiWork& w = h->fw;
    if (nnz_g) *nnz_g = w.nnz_g;
    const long nz = (long)w.nnz_g;
    if (d_X)
        features_kernel<<<g1(nz), 256, 0, s>>>(nz, w.g_row, h->G.ci, w.g_aidx, h->A.v,
                                               rinfo_of(w, (int)h->A.n_rows), w.X, d_X);
    if (d_g_row_ptr)
        MPS_CUDA(cudaMemcpyAsync(d_g_row_ptr, h->G.rp, ((size_t)h->A.n_rows + 1) * 4, cudaMemcpyDefault, s));
    if (d_g_col_ind) MPS_CUDA(cudaMemcpyAsync(d_g_col_ind, h->G.ci, (size_t)nz * 4, cudaMemcpyDefault, s));
    MPS_CUDA(cudaStreamSynchronize(s));
    return MPS_OK;
}

mps_status mps_fsai_g_values(mps_csr* h, float* d_g_vals, cudaStream_t s) {
    if (!h || !d_g_vals || !h->fw.ready) return fail(MPS_ERR_ARG, "no FSAI factor on this matrix");
    MPS_CUDA(cudaMemcpyAsync(d_g_vals, h->G.v, h->fw.nnz_g * 4, cudaMemcpyDefault, s));
    return MPS_OK;
}

// Raw network passes on caller features (FP32 [N][16], rounded to BF16 here).
mps_status mps_fsai_mlp_forward(const mps_fsai_model* m, const float* d_X, uint64_t N, float* d_out,
                                cudaStream_t s) {
    if (!m || !d_X || !d_out) return fail(MPS_ERR_ARG, "null argument");
    __nv_bfloat16* xb = nullptr;
    MPS_CUDA(stream_alloc(&xb, (N + 1) * kNF * 2, s));
    MPS_CUDA(to_bf16_launch(d_X, xb, N * kNF, s));
    MPS_CUDA(mlp_forward_launch(m->packed, xb, (long)N, d_out, m->err, s));
    cudaFreeAsync(xb, s);
    return model_error(m, s);
}

mps_status mps_fsai_mlp_forward_bf16(const mps_fsai_model* m, const void* d_Xbf16, uint64_t N,
                                     float* d_out, cudaStream_t s) {
    if (!m || !d_Xbf16 || !d_out) return fail(MPS_ERR_ARG, "null argument");
    if (reinterpret_cast<uintptr_t>(d_Xbf16) & 15) return fail(MPS_ERR_ARG, "X must be 16-byte aligned");
    if (N == 0) return MPS_OK;
    MPS_CUDA(mlp_forward_launch(m->packed, static_cast<const __nv_bfloat16*>(d_Xbf16), (long)N, d_out,
                                m->err, s));
    return MPS_OK;
}

mps_status mps_fsai_mlp_backward_bf16(const mps_fsai_model* m, const void* d_Xbf16, const float* d_dout,
                                      uint64_t N, float* d_grad, cudaStream_t s) {
    if (!m || !d_Xbf16 || !d_dout || !d_grad) return fail(MPS_ERR_ARG, "null argument");
    if (reinterpret_cast<uintptr_t>(d_Xbf16) & 15) return fail(MPS_ERR_ARG, "X must be 16-byte aligned");
    MPS_CUDA(cudaMemsetAsync(d_grad, 0, kNParam * 4, s));
    if (N == 0) return MPS_OK;
    MPS_CUDA(mlp_backward_launch(m->packed, static_cast<const __nv_bfloat16*>(d_Xbf16), d_dout, (long)N,
                                 d_grad, m->err, s));
    return MPS_OK;
}

mps_status mps_fsai_model_status(const mps_fsai_model* m, cudaStream_t s) {
    if (!m) return fail(MPS_ERR_ARG, "null argument");
    return model_error(m, s);
}

mps_status mps_fsai_mlp_backward(const mps_fsai_model* m, const float* d_X, const float* d_dout,
                                 uint64_t N, float* d_grad, cudaStream_t s) {
    if (!m || !d_X || !d_dout || !d_grad) return fail(MPS_ERR_ARG, "null argument");
    __nv_bfloat16* xb = nullptr;
    MPS_CUDA(stream_alloc(&xb, (N + 1) * kNF * 2, s));
    MPS_CUDA(to_bf16_launch(d_X, xb, N * kNF, s));
    MPS_CUDA(cudaMemsetAsync(d_grad, 0, kNParam * 4, s));
    MPS_CUDA(mlp_backward_launch(m->packed, xb, d_dout, (long)N, d_grad, m->err, s));
    cudaFreeAsync(xb, s);
    return model_error(m, s);
}

// dL/dg for the factor attached to h (network values or set_fsai values are
// not distinguished): probes V (k x n, device) ; *loss = L.
static mps_status probe_grad(mps_csr* h, const float* V, int k, uint64_t seed, int n_rand,
                             float* grad_g, double* loss, cudaStream_t s) {
    FsaiWork& w = h->fw;
    const int n = (int)h->A.n_rows;
    const long nz = (long)w.nnz_g;
    MPS_CUDA(h->H.ensure(n, s));
    float* v = w.vec;
    float* u = v + (n + 4);
    float* ww = u + (n + 4);
    float* e = ww + (n + 4);
    float* t = e + (n + 4);
    float* ss = t + (n + 4);
    MPS_CUDA(cudaMemsetAsync(grad_g, 0, (size_t)nz * 4, s));
    MPS_CUDA(cudaMemsetAsync(w.d_loss, 0, 8, s));
    CsrOp A{&h->A, nullptr}, G{&h->G, nullptr}, Gt{&h->Gt, nullptr};
    double* part = h->H.ws.partials;
    unsigned* ctr = h->H.ws.counters + 15;
    for (int p = 0; p < k + n_rand; ++p) {
        if (p < n_rand) {
            rademacher_kernel<<<g1(n), 256, 0, s>>>(n, seed * 1315423911ull + (uint64_t)p, v);
        } else {
            MPS_CUDA(cudaMemcpyAsync(v, V + (size_t)(p - n_rand) * n, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
        }
        MPS_CUDA(Gt.apply(v, EpiStore{u}, s));
        MPS_CUDA(A.apply(u, EpiStore{ww}, s));
        MPS_CUDA(G.apply(ww, EpiProbeE{e, v, w.d_loss, ctr, part}, s));
        MPS_CUDA(Gt.apply(e, EpiStore{t}, s));
        MPS_CUDA(A.apply(t, EpiStore{ss}, s));
        grad_accum_kernel<<<g1(nz), 256, 0, s>>>(nz, w.g_row, h->G.ci, e, ww, v, ss, grad_g);
    }
    const double sc = 1.0 / ((double)(k + n_rand) * (double)n);
    scale_kernel<<<g1(nz), 256, 0, s>>>(nz, grad_g, nullptr, (float)(2.0 * sc));
    MPS_CUDA(cudaGetLastError());
    double l = 0;
    MPS_CUDA(cudaMemcpyAsync(&l, w.d_loss, 8, cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = l * sc;
    return MPS_OK;
}

mps_status mps_fsai_probe_grad(mps_csr* h, const float* d_V, int32_t k, float* d_grad_g, double* loss,
                               cudaStream_t s) {
    if (!h || !d_V || k <= 0 || !d_grad_g || !h->fw.ready || !h->has_fsai)
        return fail(MPS_ERR_ARG, "probe_grad needs probes and an attached network factor");
    return probe_grad(h, d_V, k, 0, 0, d_grad_g, loss, s);
}

mps_status mps_fsai_train_step(mps_fsai_model* m, mps_csr* h, int32_t n_probes, const float* d_extra,
                               int32_t n_extra, float lr, uint64_t seed, double* loss, cudaStream_t s) {
    if (!m || !h || n_probes < 0 || n_extra < 0 || n_probes + n_extra == 0 || (n_extra && !d_extra))
        return fail(MPS_ERR_ARG, "train_step: bad arguments");
    mps_status st = fsai_prepare(h, s);
    if (st != MPS_OK) return st;
    st = fsai_values(h, m, s);
    if (st != MPS_OK) return st;
    FsaiWork& w = h->fw;
    const long nz = (long)w.nnz_g;
    st = probe_grad(h, d_extra, n_extra, seed, n_probes, w.grad, loss, s);
    if (st != MPS_OK) return st;
    scale_kernel<<<g1(nz), 256, 0, s>>>(nz, w.grad, w.dgdo, 1.0f);       // dL/dout
    MPS_CUDA(cudaMemsetAsync(m->grad, 0, kNParam * 4, s));
    MPS_CUDA(mlp_backward_launch(m->packed, w.X, w.grad, nz, m->grad, m->err, s));
    m->step += 1;
    const float c1 = 1.0f / (1.0f - std::pow(0.9f, (float)m->step));
    const float c2 = 1.0f / (1.0f - std::pow(0.999f, (float)m->step));
    adam_kernel<<<(kNParam + 255) / 256, 256, 0, s>>>(m->params, m->grad, m->m, m->v, kNParam, lr, c1, c2);
    pack_kernel<<<16, 256, 0, s>>>(m->params, m->packed);
    MPS_CUDA(cudaGetLastError());
    h->has_fsai = true;   // G now holds the pre-step network's factor
    st = model_error(m, s);
    if (st != MPS_OK) return st;
    return fsai_factor_changed(h, s);
}

}  // extern "C"
