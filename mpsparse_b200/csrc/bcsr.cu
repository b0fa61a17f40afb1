// bcsr.cu -- BCSR handles: construction (pre-built arrays or GPU COO->BCSR),
// tile plans, SpMV and the CG / BiCGSTAB entry points.
#include "bcsr_kernels.cuh"
#include "driver.hpp"

namespace mps {

cudaError_t exclusive_scan_rows(const unsigned* counts, uint64_t n, int32_t* out, unsigned* bsum,
                                cudaStream_t s);

struct BcsrMat {
    int32_t* rp = nullptr;
    int32_t* ci = nullptr;
    float* v = nullptr;
    uint32_t nbr = 0, nbc = 0, B = 4;
    uint64_t nb = 0;
    uint32_t n_rows = 0, n_cols = 0, padded = 0;
    int ntiles = 0, grid = 0, cap_blocks = 0;
    int* d_tile_brow = nullptr;
    unsigned* d_err = nullptr;
    BcsrDev view() const {
        return BcsrDev{rp, ci, v, d_tile_brow, (int)nbr, ntiles, cap_blocks, d_err};
    }
    size_t smem() const { return 2 * (size_t)cap_blocks * B * B * sizeof(float); }
};

namespace {

__global__ void plan_btiles_kernel(const int* __restrict__ rp, int nbr, int T, int ntiles,
                                   int* __restrict__ tile_brow) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > ntiles) return;
    if (t == 0) { tile_brow[0] = 0; return; }
    if (t == ntiles) { tile_brow[t] = nbr; return; }
    const long long target = (long long)t * T;
    int lo = 0, hi = nbr;
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (rp[mid] < target) lo = mid + 1; else hi = mid;
    }
    tile_brow[t] = lo;
}

// COO -> BCSR, step 1: block keys (row/B << 32 | col/B), payload = entry index;
// also the range check of the scalar keys.
__global__ void block_keys_kernel(const unsigned long long* __restrict__ keys, uint64_t nnz, int B,
                                  uint32_t n_rows, uint32_t n_cols,
                                  unsigned long long* __restrict__ bkeys, unsigned* __restrict__ idx,
                                  unsigned* err) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        const uint32_t r = (uint32_t)(k >> 32), c = (uint32_t)k;
        if (r >= n_rows || c >= n_cols) atomicOr(err, kErrRange);
        bkeys[i] = ((unsigned long long)(r / B) << 32) | (c / B);
        idx[i] = (unsigned)i;
    }
}

// Step 2: distinct block columns per block row (entries are sorted by block
// column inside each block row).
__global__ void count_blocks_kernel(const int* __restrict__ erp, const int* __restrict__ ebc,
                                    int nbr, unsigned* __restrict__ cnt) {
    for (int br = blockIdx.x * blockDim.x + threadIdx.x; br < nbr; br += gridDim.x * blockDim.x) {
        unsigned c = 0;
        for (int i = erp[br]; i < erp[br + 1]; ++i)
            if (i == erp[br] || ebc[i] != ebc[i - 1]) ++c;
        cnt[br] = c;
    }
}

// Step 3: block col_ind and densified values (duplicates summed in input order).
__global__ void fill_blocks_kernel(const int* __restrict__ erp, const int* __restrict__ ebc,
                                   const unsigned* __restrict__ eidx,
                                   const unsigned long long* __restrict__ keys,
                                   const float* __restrict__ vals, int nbr, int B,
                                   const int* __restrict__ brp, int* __restrict__ bci,
                                   float* __restrict__ bv) {
    for (int br = blockIdx.x * blockDim.x + threadIdx.x; br < nbr; br += gridDim.x * blockDim.x) {
        int slot = brp[br] - 1;
        for (int i = erp[br]; i < erp[br + 1]; ++i) {
            if (i == erp[br] || ebc[i] != ebc[i - 1]) {
                ++slot;
                bci[slot] = ebc[i];
            }
            const unsigned e = eidx[i];
            const unsigned long long k = keys[e];
            const uint32_t r = (uint32_t)(k >> 32) % B, c = (uint32_t)k % B;
            bv[(size_t)slot * B * B + r * B + c] += vals[e];
        }
    }
}

template <int B, class Epi>
cudaError_t bcsr_apply(const BcsrMat& A, const float* x, const Epi& e, cudaStream_t s) {
    const size_t smem = A.smem();
    smem_optin_k(bcsr_tiles<B, Epi>, smem);
    bcsr_tiles<B, Epi><<<A.grid, kNT, smem, s>>>(A.view(), x, e);
    return cudaGetLastError();
}

int grid1(uint64_t n) {
    uint64_t g = (n + 255) / 256, c = (uint64_t)num_sms() * 8;
    return (int)(g < 1 ? 1 : (g > c ? c : g));
}

// *out = ||b - A x||^2 in FP64 (the true residual of a returned x): one
// thread per scalar row, exact FP64 products of the FP32 block values and x,
// FP64 sums, per-CTA partials summed in a fixed order by the last CTA.
template <int B>
__global__ void __launch_bounds__(kNT)
bcsr_true_resid(const int* __restrict__ rp, const int* __restrict__ ci, const float* __restrict__ v,
                int nbr, const float* __restrict__ x, const float* __restrict__ b, double* out,
                unsigned* ctr, double* part) {
    __shared__ double red[kNT / 32];
    __shared__ int last;
    double acc = 0.0;
    const int n = nbr * B;
    for (int row = blockIdx.x * kNT + threadIdx.x; row < n; row += gridDim.x * kNT) {
        const int br = row / B, k = row % B;
        double s = 0.0;
        for (int j = rp[br]; j < rp[br + 1]; ++j) {
            const float* a = v + (size_t)j * B * B + k * B;
            const float* xs = x + (size_t)ci[j] * B;
#pragma unroll
            for (int c = 0; c < B; ++c) s += (double)a[c] * (double)xs[c];
        }
        const double r = (double)b[row] - s;
        acc += r * r;
    }
    const double t = block_sum<kNT>(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
    if (!arrive_last(ctr, &last)) return;
    const double tot = sum_partials<kNT>(part, gridDim.x, red);
    if (threadIdx.x == 0) *out = tot;
}

}  // namespace

// BCSR operator for the shared solver driver.
struct BcsrOp {
    const BcsrMat* A;
    template <class Epi>
    cudaError_t apply(const float* x, const Epi& e, cudaStream_t s) const {
        return A->B == 8 ? bcsr_apply<8>(*A, x, e, s) : bcsr_apply<4>(*A, x, e, s);
    }
    cudaError_t true_resid(const float* x, const float* b, double* out, unsigned* ctr, double* part,
                           cudaStream_t s) const {
        const int g = grid1((uint64_t)A->nbr * A->B);
        if (A->B == 8)
            bcsr_true_resid<8><<<g, kNT, 0, s>>>(A->rp, A->ci, A->v, (int)A->nbr, x, b, out, ctr, part);
        else
            bcsr_true_resid<4><<<g, kNT, 0, s>>>(A->rp, A->ci, A->v, (int)A->nbr, x, b, out, ctr, part);
        return cudaGetLastError();
    }
};

cudaError_t bcsr_plan(BcsrMat& A, cudaStream_t s) {
    const double avg = A.nbr ? (double)A.nb / A.nbr : 1.0;
    const int rows_per_tile = kNT / (int)A.B;                  // one thread per scalar row
    int T = (int)(rows_per_tile * (avg < 1.0 ? 1.0 : avg) + 0.5);
    const int cap_max = (int)((96 * 1024) / (A.B * A.B * sizeof(float)));   // per buffer
    if (T > cap_max - 32) T = cap_max - 32;
    if (T < 8) T = 8;
    A.cap_blocks = T + 32 < cap_max ? T + 32 : cap_max;
    A.ntiles = A.nb ? (int)((A.nb + T - 1) / T) : 1;
    const int cap_grid = num_sms() * 2;
    A.grid = A.ntiles < cap_grid ? A.ntiles : cap_grid;
    if (A.d_tile_brow) cudaFree(A.d_tile_brow);
    cudaError_t e = cudaMalloc(&A.d_tile_brow, (size_t)(A.ntiles + 1) * sizeof(int));
    if (e != cudaSuccess) return e;
    plan_btiles_kernel<<<(A.ntiles + 256) / 256, 256, 0, s>>>(A.rp, (int)A.nbr, T, A.ntiles,
                                                              A.d_tile_brow);
    return cudaGetLastError();
}

}  // namespace mps

using namespace mps;

struct mps_bcsr {
    BcsrMat A;
    SolverHost H;
};

static void bcsr_free(BcsrMat& m) {
    if (m.rp) cudaFree(m.rp);
    if (m.ci) cudaFree(m.ci);
    if (m.v) cudaFree(m.v);
    if (m.d_tile_brow) cudaFree(m.d_tile_brow);
    if (m.d_err) cudaFree(m.d_err);
    m = BcsrMat{};
}

static mps_status bcsr_shape_init(BcsrMat& A, uint32_t n_rows, uint32_t n_cols, uint32_t block,
                                  uint64_t nb) {
    if (block != 4 && block != 8) return fail(MPS_ERR_ARG, "block size must be 4 or 8");
    if (n_rows == 0 || n_cols == 0) return fail(MPS_ERR_ARG, "num_rows and num_cols must be positive");
    if (n_rows != n_cols) return fail(MPS_ERR_ARG, "BCSR solvers need a square matrix");
    A.B = block;
    A.n_rows = n_rows;
    A.n_cols = n_cols;
    A.nbr = (n_rows + block - 1) / block;
    A.nbc = (n_cols + block - 1) / block;
    A.padded = A.nbr * block;
    A.nb = nb;
    if (nb >= 0x7fffff00ull) return fail(MPS_ERR_ARG, "too many blocks");
    MPS_CUDA(cudaMalloc(&A.rp, ((size_t)A.nbr + 1) * 4));
    MPS_CUDA(cudaMalloc(&A.ci, (nb ? nb : 1) * 4));
    MPS_CUDA(cudaMalloc(&A.v, (nb ? nb : 1) * block * block * 4));
    MPS_CUDA(cudaMalloc(&A.d_err, 4));
    MPS_CUDA(cudaMemset(A.d_err, 0, 4));
    return MPS_OK;
}

extern "C" {

mps_status mps_bcsr_create(const float* d_vals, const int32_t* d_row_ptr, const int32_t* d_col_ind,
                           uint64_t n_blocks, uint32_t n_rows, uint32_t n_cols, uint32_t block,
                           mps_bcsr** out, cudaStream_t s) {
    if (!out || !d_row_ptr || (n_blocks && (!d_vals || !d_col_ind)))
        return fail(MPS_ERR_ARG, "null argument");
    *out = nullptr;
    mps_bcsr* h = new mps_bcsr();
    mps_status st = bcsr_shape_init(h->A, n_rows, n_cols, block, n_blocks);
    if (st != MPS_OK) {
        mps_bcsr_destroy(h);
        return st;
    }
    BcsrMat& A = h->A;
    MPS_CUDA(cudaMemcpyAsync(A.rp, d_row_ptr, ((size_t)A.nbr + 1) * 4, cudaMemcpyDeviceToDevice, s));
    if (n_blocks) {
        MPS_CUDA(cudaMemcpyAsync(A.ci, d_col_ind, n_blocks * 4, cudaMemcpyDeviceToDevice, s));
        MPS_CUDA(cudaMemcpyAsync(A.v, d_vals, n_blocks * block * block * 4, cudaMemcpyDeviceToDevice, s));
    }
    cudaError_t e = bcsr_plan(A, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        mps_bcsr_destroy(h);
        return cuda_fail(e, "bcsr_create");
    }
    *out = h;
    return MPS_OK;
}

mps_status mps_bcsr_create_from_keys(const uint64_t* d_keys, const float* d_vals, uint64_t nnz,
                                     uint32_t n_rows, uint32_t n_cols, uint32_t block,
                                     mps_bcsr** out, cudaStream_t s) {
    if (!out || (nnz && (!d_keys || !d_vals))) return fail(MPS_ERR_ARG, "null argument");
    *out = nullptr;
    if (block != 4 && block != 8) return fail(MPS_ERR_ARG, "block size must be 4 or 8");
    if (nnz >= 0x7fffff00ull) return fail(MPS_ERR_ARG, "nnz must be < 2^31");
    const uint32_t nbr = (n_rows + block - 1) / block, nbc = (n_cols + block - 1) / block;
    // Temporaries: block keys, entry index, entry row_ptr / block col / index.
    unsigned long long* bkeys = nullptr;
    unsigned *idx = nullptr, *eidx = nullptr, *cnt = nullptr, *bsum = nullptr, *d_err = nullptr;
    int *erp = nullptr, *ebc = nullptr;
    const size_t nz = nnz ? nnz : 1;
    MPS_CUDA(stream_alloc(&bkeys, nz * 8, s));
    MPS_CUDA(stream_alloc(&idx, nz * 4, s));
    MPS_CUDA(stream_alloc(&eidx, nz * 4, s));
    MPS_CUDA(stream_alloc(&ebc, nz * 4, s));
    MPS_CUDA(stream_alloc(&erp, ((size_t)nbr + 1) * 4, s));
    MPS_CUDA(stream_alloc(&cnt, ((size_t)nbr + 1) * 4, s));
    MPS_CUDA(stream_alloc(&bsum, (((size_t)nbr + 2048) / 2048 + 1) * 4, s));
    MPS_CUDA(stream_alloc(&d_err, 4, s));
    MPS_CUDA(cudaMemsetAsync(d_err, 0, 4, s));
    int* brp = nullptr;
    MPS_CUDA(stream_alloc(&brp, ((size_t)nbr + 1) * 4, s));
    if (nnz)
        block_keys_kernel<<<grid1(nnz), 256, 0, s>>>(reinterpret_cast<const unsigned long long*>(d_keys),
                                                      nnz, (int)block, n_rows, n_cols, bkeys, idx, d_err);
    MPS_CUDA(cudaGetLastError());
    MPS_CUDA(sort_to_csr(reinterpret_cast<const uint64_t*>(bkeys), idx, nnz, nbr, nbc, erp, ebc, eidx,
                         d_err, s));
    count_blocks_kernel<<<grid1(nbr), 256, 0, s>>>(erp, ebc, (int)nbr, cnt);
    MPS_CUDA(exclusive_scan_rows(cnt, nbr, brp, bsum, s));
    int nb_i = 0;
    unsigned err = 0;
    MPS_CUDA(cudaMemcpyAsync(&nb_i, brp + nbr, 4, cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaMemcpyAsync(&err, d_err, 4, cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaStreamSynchronize(s));
    mps_status st = MPS_OK;
    mps_bcsr* h = nullptr;
    if (err & kErrRange)
        st = fail(MPS_ERR_RANGE, "bcsr: a key lies outside [0, num_rows) x [0, num_cols)");
    else if (err & kErrTimeout)
        st = fail(MPS_ERR_TIMEOUT, "bcsr: a bounded device wait gave up");
    if (st == MPS_OK) {
        h = new mps_bcsr();
        st = bcsr_shape_init(h->A, n_rows, n_cols, block, (uint64_t)nb_i);
    }
    if (st == MPS_OK) {
        BcsrMat& A = h->A;
        cudaError_t e = cudaMemcpyAsync(A.rp, brp, ((size_t)nbr + 1) * 4, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(A.v, 0, (size_t)(nb_i ? nb_i : 1) * block * block * 4, s);
        if (e == cudaSuccess) {
            fill_blocks_kernel<<<grid1(nbr), 256, 0, s>>>(erp, ebc, eidx,
                                                          reinterpret_cast<const unsigned long long*>(d_keys),
                                                          d_vals, (int)nbr, (int)block, brp, A.ci, A.v);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = bcsr_plan(A, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "bcsr_create_from_keys");
    }
    cudaFreeAsync(bkeys, s);
    cudaFreeAsync(idx, s);
    cudaFreeAsync(eidx, s);
    cudaFreeAsync(ebc, s);
    cudaFreeAsync(erp, s);
    cudaFreeAsync(cnt, s);
    cudaFreeAsync(bsum, s);
    cudaFreeAsync(d_err, s);
    cudaFreeAsync(brp, s);
    if (st != MPS_OK) {
        if (h) mps_bcsr_destroy(h);
        return st;
    }
    *out = h;
    return MPS_OK;
}

mps_status mps_bcsr_destroy(mps_bcsr* h) {
    if (!h) return MPS_OK;
    bcsr_free(h->A);
    h->H.destroy();
    delete h;
    return MPS_OK;
}

mps_status mps_bcsr_shape(const mps_bcsr* h, uint32_t* nbr, uint64_t* nb, uint32_t* block,
                          uint32_t* padded) {
    if (!h) return fail(MPS_ERR_ARG, "null handle");
    if (nbr) *nbr = h->A.nbr;
    if (nb) *nb = h->A.nb;
    if (block) *block = h->A.B;
    if (padded) *padded = h->A.padded;
    return MPS_OK;
}

mps_status mps_bcsr_export(const mps_bcsr* h, int32_t* rp, int32_t* ci, float* v, cudaStream_t s) {
    if (!h) return fail(MPS_ERR_ARG, "null handle");
    const BcsrMat& A = h->A;
    if (rp) MPS_CUDA(cudaMemcpyAsync(rp, A.rp, ((size_t)A.nbr + 1) * 4, cudaMemcpyDefault, s));
    if (ci && A.nb) MPS_CUDA(cudaMemcpyAsync(ci, A.ci, A.nb * 4, cudaMemcpyDefault, s));
    if (v && A.nb) MPS_CUDA(cudaMemcpyAsync(v, A.v, A.nb * A.B * A.B * 4, cudaMemcpyDefault, s));
    return MPS_OK;
}

mps_status mps_bcsr_spmv(const mps_bcsr* h, const float* x, float* y, cudaStream_t s) {
    if (!h || !x || !y) return fail(MPS_ERR_ARG, "null argument");
    BcsrOp op{&h->A};
    MPS_CUDA(op.apply(x, EpiStore{y}, s));
    return MPS_OK;
}

static mps_status bcsr_solve(SolverKind kind, mps_bcsr* h, const float* b, float* x,
                             const mps_solve_opts* o, mps_solve_info* info, cudaStream_t s) {
    if (!h || !b || !x) return fail(MPS_ERR_ARG, "null argument");
    mps_solve_opts oo;
    mps_solve_opts_default(&oo);
    if (o) oo = *o;
    oo.precond = MPS_PRECOND_NONE;
    MPS_CUDA(h->H.ensure(h->A.padded, s));
    MPS_CUDA(cudaMemsetAsync(h->A.d_err, 0, 4, s));
    BcsrOp op{&h->A};
    PrecondOps<BcsrOp> pc{};
    mps_status st = run_solve(kind, op, pc, h->H, b, x, &oo, info, s);
    unsigned err = 0;
    MPS_CUDA(cudaMemcpy(&err, h->A.d_err, 4, cudaMemcpyDeviceToHost));
    if (st == MPS_OK && (err & kErrTimeout)) return fail(MPS_ERR_TIMEOUT, "bcsr: bulk-copy wait gave up");
    return st;
}

mps_status mps_bcsr_cg(mps_bcsr* h, const float* b, float* x, const mps_solve_opts* o,
                       mps_solve_info* info, cudaStream_t s) {
    return bcsr_solve(kCG, h, b, x, o, info, s);
}

mps_status mps_bcsr_bicgstab(mps_bcsr* h, const float* b, float* x, const mps_solve_opts* o,
                             mps_solve_info* info, cudaStream_t s) {
    return bcsr_solve(kBiCG, h, b, x, o, info, s);
}

}  // extern "C"
