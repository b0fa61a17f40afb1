/*
 * oracle.h -- CPU restatement of SparseForge/mpsparse's sparse iterative-solver
 * path.  TEST INFRASTRUCTURE ONLY: this library is the checker that the CUDA
 * path is compared against.  It is loaded by tests/, by __graft_entry__.smoke()
 * and by bench.py's CPU-baseline leg, never by the product path.
 *
 * Parity status: the sort/CSR build and the SpMV are pinned by the reference's
 * own ground-truth checks (torch.to_sparse_csr and torch CSR mm, as used in
 * spmv_kernel/coo_csr/coo_csr/coo_csr/benchmark.py:133-156 and
 * spmv_kernel/spmv/benchmark.py:172-177), re-run here as golden fixtures.  The
 * solver iterates are pinned against scipy's independent CG/BiCGSTAB iterates
 * (tests/golden); the reference itself ships no golden vectors and cannot run
 * here (Metal), so the reference_compat quirks are "parity unpinned".
 */
#ifndef MPS_ORACLE_H
#define MPS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Stable masked 4-bit LSD sort of packed (row<<32|col) keys with float payload,
 * followed by the compress + row-fixer CSR build.
 * Follows iterative/BiCGSTAB/spmv.cpp:62-228 and coo_csr.metal:17-193. */
int orc_coo_to_csr(const uint64_t* keys, const float* vals, uint64_t nnz,
                   uint32_t n_rows, uint32_t n_cols,
                   int32_t* row_ptr, int32_t* col_ind, float* out_vals);

/* y = A x, FP64 accumulation over FP32 values (spmv.metal:11-49). */
void orc_csr_spmv(const int32_t* row_ptr, const int32_t* col_ind, const float* val,
                  int64_t n_rows, const double* x, double* y, int threads);

/* y = A x for 4x4 row-major BCSR blocks (bcsr_spmv.metal:30-69), any block size. */
void orc_bcsr_spmv(const int32_t* row_ptr, const int32_t* col_ind, const float* val,
                   int64_t n_block_rows, int block, const double* x, double* y);

/* Solver options.  compat=1 reproduces the reference's quirks (x0 = 0, the
 * iteration caps, the absolute squared-norm test every 50 iterations, the
 * BiCGSTAB rho0 = 1 + r.r start); compat=0 is the plain algorithm with a
 * relative residual test ||r|| <= tol ||b|| on every iteration. */
typedef struct {
    int compat;
    int max_iter;        /* compat=0: iteration cap */
    double tol;          /* compat=0: relative residual target */
    double omega;        /* Richardson weight */
    int threads;         /* OpenMP threads for the SpMV/dots (1 = serial) */
    int precond;         /* 0 none, 1 Jacobi (CG only) */
} orc_opts;

typedef struct {
    int iters;
    int converged;
    int breakdown;
    double rel_resid;    /* recurrence residual ||r||/||b|| at exit */
} orc_info;

/* Operator descriptor: CSR (block = 0) or BCSR (block = 4 or 8). */
typedef struct {
    const int32_t* row_ptr;
    const int32_t* col_ind;
    const float* val;
    int64_t n;           /* scalar rows (padded for BCSR) */
    int block;
} orc_op;

/* CG: iterative/BiCGSTAB/spmv.cpp:528-659 with cgd.metal:11-82. */
int orc_cg(const orc_op* A, const double* b, double* x, const orc_opts* o, orc_info* info);
/* BiCGSTAB: iterative/BiCGSTAB/spmv.cpp:699-888 with bicgstab.metal:12-326. */
int orc_bicgstab(const orc_op* A, const double* b, double* x, const orc_opts* o, orc_info* info);
/* Richardson: iterative/richardson/spmv.cpp:376-495 with spmv.metal:50-63. */
int orc_richardson(const orc_op* A, const double* b, double* x, const orc_opts* o, orc_info* info);

/* ||b - A x|| / ||b|| in FP64. */
double orc_true_residual(const orc_op* A, const double* b, const double* x);

/* ---- learned FSAI preconditioner (no reference counterpart) -------------- */
#define ORC_NF 16
#define ORC_NH 64
/* parameter vector: W1[16][64], b1[64], W2[64][64], b2[64], w3[64], b3 */
#define ORC_NPARAM (ORC_NF * ORC_NH + ORC_NH + ORC_NH * ORC_NH + ORC_NH + ORC_NH + 1)

/* Lower-triangular pattern of A (cols <= row); returns nnz(G).  Arrays are
 * sized by the caller: g_rp[n+1], the others nnz(A). */
int64_t orc_fsai_pattern(const orc_op* A, int32_t* g_rp, int32_t* g_ci, int32_t* g_row,
                         int32_t* g_aidx);
/* 16 features per G nonzero (row-major X[nnzG][16]). */
void orc_fsai_features(const orc_op* A, int64_t nnz_g, const int32_t* g_row, const int32_t* g_ci,
                       const int32_t* g_aidx, float* X);
/* MLP 16->64->64->1 (GELU) with the device's rounding points: features,
 * W1, W2, w3 and the first hidden layer in BF16, FP64 accumulation here. */
void orc_mlp_forward(const float* params, const float* X, int64_t N, double* out);
/* Parameter gradient for dL/dout (same rounding points as the device:
 * dz2 and dz1 rounded to BF16 before the weight-gradient products). */
void orc_mlp_backward(const float* params, const float* X, int64_t N, const double* dout,
                      double* grad);
/* Probe estimate L = sum_v ||v - G A G^T v||^2 / (k n) and dL/dG on G's
 * pattern.  V is k x n row-major. */
double orc_fsai_probe_loss_grad(const orc_op* A, const orc_op* G, const double* V, int k,
                                double* grad_g);

#ifdef __cplusplus
}
#endif
#endif
