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

#ifdef __cplusplus
}
#endif
#endif
