// fsai_product.cu -- M = G^T G for the FSAI preconditioner.
//
// PCG with an FSAI factor applies z = G^T (G r): two SpMVs and two kernel
// launches per iteration.  On systems small enough for the solve to be bound
// by launch and reduction latency rather than by bytes (every vector and
// matrix of a 512^2 system fits in L2), one SpMV with M = G^T G is faster,
// although M holds more nonzeros than G and G^T together (7 versus 6 per row
// for a 5-point stencil).  The choice per matrix (auto) weighs one launch
// against the extra bytes of M.
//
// Construction, on the GPU, one thread per row i of M (rows of G^T G are
// short for the sparse factors this targets):
//   pattern (once per pattern of G): for each k of row i of G^T (g_ki != 0)
//   and each nonzero g_kj of row k of G, the pair (g_ki, g_kj) is inserted
//   into a per-thread list sorted by j (stable, so ascending k among equal
//   j); a count pass sizes M and the pair list, a fill pass writes M's
//   columns and, per nonzero, the range of its pairs;
//   values (after every change of G's values): m_ij = sum over the range of
//   g_ki g_kj, summed in FP64 in ascending k, so M is exactly symmetric.
#include <cstring>

#include "handles.hpp"

namespace mps {

namespace {

constexpr int kPNT = 256;
inline int grid_for(uint64_t n) {
    uint64_t g = (n + kPNT - 1) / kPNT;
    const uint64_t cap = (uint64_t)num_sms() * 8;
    if (g > cap) g = cap;
    return g < 1 ? 1 : (int)g;
}

// Candidate pairs per row of M held by one thread; rows with more make the
// product form unavailable (auto keeps the split form).
constexpr int kRowCap = 96;

// Index of g_ki (column i in row k of G), or -1.
__device__ __forceinline__ int find_in_row(const int32_t* __restrict__ grp, const int32_t* __restrict__ gci,
                                           int k, int i) {
    for (int a = grp[k]; a < grp[k + 1]; ++a)
        if (gci[a] == i) return a;
    return -1;
}

// Row i of M: candidate pairs sorted by column (stable).  Returns the count,
// or -1 when the row holds more than kRowCap pairs.
__device__ __forceinline__ int row_pairs(const int32_t* __restrict__ grp, const int32_t* __restrict__ gci,
                                         const int32_t* __restrict__ trp, const int32_t* __restrict__ tci,
                                         int i, int* cols, int* ia, int* ib) {
    int nc = 0;
    for (int t = trp[i]; t < trp[i + 1]; ++t) {
        const int k = tci[t];
        const int a = find_in_row(grp, gci, k, i);
        if (a < 0) continue;
        for (int b = grp[k]; b < grp[k + 1]; ++b) {
            if (nc == kRowCap) return -1;
            const int c = gci[b];
            int q = nc++;
            while (q > 0 && cols[q - 1] > c) {   // insert after equal columns
                cols[q] = cols[q - 1];
                if (ia) {
                    ia[q] = ia[q - 1];
                    ib[q] = ib[q - 1];
                }
                --q;
            }
            cols[q] = c;
            if (ia) {
                ia[q] = a;
                ib[q] = b;
            }
        }
    }
    return nc;
}

__global__ void product_count_kernel(const int32_t* __restrict__ grp, const int32_t* __restrict__ gci,
                                     const int32_t* __restrict__ trp, const int32_t* __restrict__ tci, int n,
                                     unsigned* __restrict__ mcnt, unsigned* __restrict__ pcnt,
                                     unsigned* __restrict__ over) {
    int cols[kRowCap];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int nc = row_pairs(grp, gci, trp, tci, i, cols, nullptr, nullptr);
        if (nc < 0) {
            atomicOr(over, 1u);
            mcnt[i] = pcnt[i] = 0;
            continue;
        }
        unsigned u = 0;
        for (int q = 0; q < nc; ++q) u += (q == 0 || cols[q] != cols[q - 1]);
        mcnt[i] = u;
        pcnt[i] = (unsigned)nc;
    }
}

__global__ void product_fill_kernel(const int32_t* __restrict__ grp, const int32_t* __restrict__ gci,
                                    const int32_t* __restrict__ trp, const int32_t* __restrict__ tci, int n,
                                    const int32_t* __restrict__ mrp, const int32_t* __restrict__ poff,
                                    int32_t* __restrict__ mci, int32_t* __restrict__ seg,
                                    int32_t* __restrict__ pa, int32_t* __restrict__ pb) {
    int cols[kRowCap], ia[kRowCap], ib[kRowCap];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int nc = row_pairs(grp, gci, trp, tci, i, cols, ia, ib);
        if (nc < 0) continue;   // the count pass reported it
        int m = mrp[i];
        const int p0 = poff[i];
        for (int q = 0; q < nc; ++q) {
            pa[p0 + q] = ia[q];
            pb[p0 + q] = ib[q];
            if (q == 0 || cols[q] != cols[q - 1]) {
                mci[m] = cols[q];
                seg[m] = p0 + q;
                ++m;
            }
        }
        if (i == n - 1) seg[mrp[n]] = poff[n];
    }
}

__global__ void product_values_kernel(long nnz_m, const int32_t* __restrict__ seg,
                                      const int32_t* __restrict__ pa, const int32_t* __restrict__ pb,
                                      const float* __restrict__ gv, float* __restrict__ mv) {
    for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < nnz_m; m += (long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int t = seg[m]; t < seg[m + 1]; ++t) s += (double)gv[pa[t]] * (double)gv[pb[t]];
        mv[m] = (float)s;
    }
}

// One launch saved versus the extra bytes M streams: at ~6 us per dependent
// launch and ~5 TB/s, M pays while it holds fewer than ~3.75M nonzeros more
// than G and G^T together.
constexpr uint64_t kExtraEntriesPerLaunch = 3750000;
constexpr uint64_t kMaxPairs = 0x7fffff00ull;

mps_status product_pattern(mps_csr* h, bool forced, cudaStream_t s) {
    FsaiProduct& fp = h->fp;
    const int n = (int)h->G.n_rows;
    const uint64_t nnz_g = h->G.nnz;
    if ((uint64_t)n * kRowCap >= kMaxPairs) {   // pair offsets are int32
        if (forced) return fail(MPS_ERR_ARG, "G^T G: too many rows for the product form");
        fp.declined = true;
        return MPS_OK;
    }
    const size_t nb = (size_t)n + 1;
    unsigned *mcnt = nullptr, *pcnt = nullptr, *bsum = nullptr, *over = nullptr;
    int32_t *mrp = nullptr, *poff = nullptr;
    MPS_CUDA(stream_alloc(&mcnt, nb * 4, s));
    MPS_CUDA(stream_alloc(&pcnt, nb * 4, s));
    MPS_CUDA(stream_alloc(&bsum, ((nb + 2048) / 2048 + 1) * 4, s));
    MPS_CUDA(stream_alloc(&over, 4, s));
    MPS_CUDA(stream_alloc(&mrp, nb * 4, s));
    MPS_CUDA(stream_alloc(&poff, nb * 4, s));
    auto release = [&]() {
        cudaFreeAsync(mcnt, s);
        cudaFreeAsync(pcnt, s);
        cudaFreeAsync(bsum, s);
        cudaFreeAsync(over, s);
        cudaFreeAsync(mrp, s);
        cudaFreeAsync(poff, s);
    };
    MPS_CUDA(cudaMemsetAsync(over, 0, 4, s));
    product_count_kernel<<<grid_for(n), kPNT, 0, s>>>(h->G.rp, h->G.ci, h->Gt.rp, h->Gt.ci, n, mcnt, pcnt, over);
    MPS_CUDA(cudaGetLastError());
    MPS_CUDA(exclusive_scan_rows(mcnt, n, mrp, bsum, s));
    MPS_CUDA(exclusive_scan_rows(pcnt, n, poff, bsum, s));
    int32_t tot[2] = {0, 0};
    unsigned ov = 0;
    MPS_CUDA(cudaMemcpyAsync(&tot[0], mrp + n, 4, cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaMemcpyAsync(&tot[1], poff + n, 4, cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaMemcpyAsync(&ov, over, 4, cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaStreamSynchronize(s));
    const uint64_t nnz_m = (uint64_t)tot[0], E = (uint64_t)tot[1];
    // decline: a row beyond the per-thread list, or (auto) more extra bytes
    // than one launch is worth
    if (ov || (!forced && nnz_m > 2 * nnz_g + kExtraEntriesPerLaunch)) {
        release();
        if (forced) return fail(MPS_ERR_ARG, "G^T G: a row has more than 96 products");
        fp.declined = true;
        return MPS_OK;
    }
    const size_t ez = (size_t)(E ? E : 1);
    mps_status st = alloc_csr(h->M, (uint32_t)n, (uint32_t)n, nnz_m, h->d_err, s);
    if (st == MPS_OK) {
        cudaError_t e = dev_alloc(&fp.seg, ((size_t)nnz_m + 1) * 4, s);
        if (e == cudaSuccess) e = dev_alloc(&fp.pa, ez * 4, s);
        if (e == cudaSuccess) e = dev_alloc(&fp.pb, ez * 4, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h->M.rp, mrp, nb * 4, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(fp.seg, 0, ((size_t)nnz_m + 1) * 4, s);
        if (e == cudaSuccess) {
            product_fill_kernel<<<grid_for(n), kPNT, 0, s>>>(h->G.rp, h->G.ci, h->Gt.rp, h->Gt.ci, n, mrp, poff,
                                                            h->M.ci, fp.seg, fp.pa, fp.pb);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = spmv_plan_build(h->M, 0, s, h->A.plan.stages, h->A.plan.evict_first);
        if (e != cudaSuccess) st = cuda_fail(e, "G^T G pattern");
    }
    release();
    if (st != MPS_OK) {
        fsai_product_free(h);
        return st;
    }
    fp.n_pairs = E;
    fp.ready = true;
    return MPS_OK;
}

}  // namespace

void fsai_product_free(mps_csr* h) {
    FsaiProduct& fp = h->fp;
    dev_free(fp.seg);
    dev_free(fp.pa);
    dev_free(fp.pb);
    fp = FsaiProduct{};
    persist_plan_free(h);
    csr_free(h->M);
    if (h->use_m) h->H.drop_graphs();
    h->use_m = false;
}

mps_status fsai_factor_changed(mps_csr* h, cudaStream_t s) {
    const bool before = h->use_m;
    bool want = false;
    if (h->G.rp && h->G.n_rows && h->fsai_apply != MPS_FSAI_APPLY_SPLIT) {
        const bool forced = h->fsai_apply == MPS_FSAI_APPLY_PRODUCT;
        if (forced) h->fp.declined = false;
        if (!h->fp.ready && !h->fp.declined) {
            mps_status st = product_pattern(h, forced, s);
            if (st != MPS_OK) return st;
        }
        want = h->fp.ready;
    }
    if (want) {
        const long nnz_m = (long)h->M.nnz;
        product_values_kernel<<<grid_for((uint64_t)nnz_m), kPNT, 0, s>>>(nnz_m, h->fp.seg, h->fp.pa, h->fp.pb,
                                                                        h->G.v, h->M.v);
        MPS_CUDA(cudaGetLastError());
    }
    h->use_m = want;
    if (want != before) h->H.drop_graphs();   // graphs hold one apply form
    return MPS_OK;
}

}  // namespace mps

using namespace mps;

extern "C" {

mps_status mps_csr_set_fsai_apply(mps_csr* h, int32_t mode, cudaStream_t stream) {
    if (!h) return fail(MPS_ERR_ARG, "null handle");
    if (mode != MPS_FSAI_APPLY_AUTO && mode != MPS_FSAI_APPLY_SPLIT && mode != MPS_FSAI_APPLY_PRODUCT)
        return fail(MPS_ERR_ARG, "mode must be MPS_FSAI_APPLY_AUTO, _SPLIT or _PRODUCT");
    h->fsai_apply = mode;
    if (!h->has_fsai) return MPS_OK;
    return fsai_factor_changed(h, stream);
}

mps_status mps_csr_fsai_apply(const mps_csr* h, int32_t* in_force, uint64_t* nnz_m) {
    if (!h || !in_force) return fail(MPS_ERR_ARG, "null argument");
    *in_force = !h->has_fsai ? -1 : (h->use_m ? MPS_FSAI_APPLY_PRODUCT : MPS_FSAI_APPLY_SPLIT);
    if (nnz_m) *nnz_m = h->use_m ? h->M.nnz : 0;
    return MPS_OK;
}

mps_status mps_csr_fsai_product_get(const mps_csr* h, int32_t* d_rp, int32_t* d_ci, float* d_v,
                                    cudaStream_t s) {
    if (!h || !d_rp || !d_ci || !d_v) return fail(MPS_ERR_ARG, "null argument");
    if (!h->has_fsai || !h->use_m) return fail(MPS_ERR_ARG, "no G^T G in force on this matrix");
    MPS_CUDA(cudaMemcpyAsync(d_rp, h->M.rp, ((size_t)h->M.n_rows + 1) * 4, cudaMemcpyDefault, s));
    if (h->M.nnz) {
        MPS_CUDA(cudaMemcpyAsync(d_ci, h->M.ci, h->M.nnz * 4, cudaMemcpyDefault, s));
        MPS_CUDA(cudaMemcpyAsync(d_v, h->M.v, h->M.nnz * 4, cudaMemcpyDefault, s));
    }
    return MPS_OK;
}

}  // extern "C"
