// handles.hpp -- definition of the opaque mps_csr handle, shared by the
// translation units that operate on it.
#pragma once
#include "driver.hpp"

namespace mps {

// Learned-FSAI state of one matrix: G's pattern (tril(A)) and its maps.
struct FsaiWork {
    bool ready = false;
    uint64_t nnz_g = 0;
    int32_t* g_row = nullptr;      // row of each G nonzero
    int32_t* g_aidx = nullptr;     // index of the matching entry of A
    uint32_t* perm = nullptr;      // G^T position -> G position
    __nv_bfloat16* X = nullptr;    // features [nnz_g][16]
    float* out = nullptr;          // MLP output per G nonzero
    float* dgdo = nullptr;         // d g / d out
    float* grad = nullptr;         // dL/dg, then dL/dout
    float* rinfo = nullptr;        // per-row feature inputs of A
    double* d_loss = nullptr;
    float* vec = nullptr;          // probe work vectors (6 x n)
};

// M = G^T G for the one-SpMV FSAI apply: its pattern and, per nonzero of M,
// the range of pairs (g_ki, g_kj) whose products sum to it.
struct FsaiProduct {
    bool ready = false;        // built for the current pattern of G
    bool declined = false;     // the cost model chose G and G^T for this pattern
    uint64_t n_pairs = 0;
    int32_t* seg = nullptr;    // nnz(M) + 1 offsets into pa / pb
    int32_t* pa = nullptr;     // index of g_ki in G's values, pairs sorted by (i, j, k)
    int32_t* pb = nullptr;     // index of g_kj
};

// Row blocks of the persistent FSAI-PCG form (fsai_persistent.cu): one CTA
// per SM holds its rows of A and M in shared memory.
struct PersistPlan {
    int state = 0;                 // 0 not built, 1 eligible, -1 rows do not fit
    int grid = 0;
    int rows_max = 0;              // most rows of one CTA
    size_t smem = 0;               // dynamic shared memory per CTA
    int form = 0;                  // 0 gather, 1 window (16-bit window-relative columns), 2 stream
    int* d_row_start = nullptr;    // grid + 1 row boundaries, the barrier's words, the windows
    unsigned short* d_c16 = nullptr;  // stream form: A's then M's columns relative to their CTA's window
};

}  // namespace mps

struct mps_csr {
    mps::CsrMat A;
    __nv_bfloat16* vb = nullptr;
    mps::CsrMat G, Gt;
    bool has_fsai = false;
    mps::SolverHost H;
    unsigned* d_err = nullptr;
    mps::FsaiWork fw;
    mps::CsrMat M;             // G^T G (when use_m)
    mps::FsaiProduct fp;
    int32_t fsai_apply = 0;    // MPS_FSAI_APPLY_*
    bool use_m = false;        // PCG applies z = M r (else z = G^T (G r))
    mps::PersistPlan pp;       // persistent form of reliable-update FSAI-PCG (rows of A and M)
    mps::PersistPlan pp_a;     // persistent form of plain CG / Jacobi-PCG (rows of A)
    int32_t persistent = 1;    // 1: use the persistent form when the rows fit
    int32_t persist_form = 0;  // 0: the first form that fits; 1 gather, 2 window, 3 stream: only that one
    // test hook of the persistent kernels' grid barrier (mps_test_persistent_barrier_timeout)
    uint32_t test_spin_limit = 0;   // 0: the default bound on one barrier wait
    int32_t test_silent_cta = -1;   // >= 0: that CTA skips its first arrival
};

namespace mps {
void csr_free(CsrMat& m);
mps_status alloc_csr(CsrMat& m, uint32_t n_rows, uint32_t n_cols, uint64_t nnz, unsigned* err,
                     cudaStream_t s);
mps_status build_from_keys(CsrMat& m, const uint64_t* keys, const uint32_t* payload, uint64_t nnz,
                           uint32_t n_rows, uint32_t n_cols, unsigned* d_err, cudaStream_t s, bool plan = true);
mps_status prepare_precond(mps_csr* h, const mps_solve_opts* o, cudaStream_t s);
cudaError_t exclusive_scan_rows(const unsigned* counts, uint64_t n, int32_t* out, unsigned* bsum,
                                cudaStream_t s);
void fsai_work_free(FsaiWork& w);
// Rebuild the SpMV plans of G, G^T and M with A's pipeline depth and L2 hint.
cudaError_t factor_plans_follow(mps_csr* h, cudaStream_t s);
// G^T G: drop it (G's pattern changed) / bring the apply form in line with
// h->fsai_apply and G's current values (pattern on first use, then values).
void fsai_product_free(mps_csr* h);
// Status of a device error word (range / timeout bits) after `what`.
mps_status device_error(unsigned err, const char* what);
mps_status fsai_factor_changed(mps_csr* h, cudaStream_t s);
// Persistent FSAI-PCG (fsai_persistent.cu): plan (built on first use, freed
// with M's pattern) and the solve; cudaErrorNotSupported: not eligible.
void persist_plan_free(mps_csr* h);
void persist_plan_free_all(mps_csr* h);
cudaError_t persist_solve(mps_csr* h, const double* b64, double* x64, cudaStream_t s);
cudaError_t persist_cg_solve(mps_csr* h, cudaStream_t s, const double* b64 = nullptr,
                             double* x64 = nullptr);
cudaError_t persist_bicg_solve(mps_csr* h, cudaStream_t s);
cudaError_t persist_rich_solve(mps_csr* h, cudaStream_t s);
}  // namespace mps
