/*
 * mpsparse.h -- C ABI of the B200 (sm_100a) sparse iterative-solver library.
 *
 * Drop-in boundary for SparseForge/mpsparse's PyTorch extension modules
 * `spmv` (class csr_tensor), `bcsr` (class bcsr_tensor) and `coo_csr`.  Each
 * entry point names the reference interface it replaces (path:line in the
 * reference project).
 *
 * Conventions
 *  - Every pointer argument named d_* is device memory on the current device;
 *    h_* is host memory.  Sizes are element counts.
 *  - Calls are stream-ordered on the given stream (0 = legacy default stream).
 *    Solvers synchronise that stream once, at the end, to fill *info.
 *  - A handle owns its device memory and is released by its destroy call.  A
 *    handle may not be used from two host threads at once.
 *  - Errors are returned as mps_status; nothing calls exit().  The message of
 *    the last error on the calling thread is mps_last_error_string().
 */
#ifndef MPSPARSE_H
#define MPSPARSE_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MPS_OK = 0,
    MPS_ERR_ARG = 1,        /* bad argument: null pointer, size, block size */
    MPS_ERR_CUDA = 2,       /* a CUDA runtime call failed */
    MPS_ERR_OOM = 3,        /* device allocation failed */
    MPS_ERR_TIMEOUT = 4,    /* a bounded device-side wait gave up */
    MPS_ERR_BREAKDOWN = 5,  /* solver breakdown (see mps_solve_info) */
    MPS_ERR_RANGE = 6,      /* a COO key lies outside [0,n_rows) x [0,n_cols) */
    MPS_ERR_NOT_FINITE = 7  /* right-hand side holds NaN or Inf */
} mps_status;

typedef struct mps_csr mps_csr;
typedef struct mps_bcsr mps_bcsr;

/* Preconditioners for mps_csr_cg. */
enum { MPS_PRECOND_NONE = 0, MPS_PRECOND_JACOBI = 1, MPS_PRECOND_FSAI = 2 };

typedef struct {
    int32_t reference_compat; /* 1: reproduce the reference's stop rules and
                                 guards (iteration caps min(1000,n) / min(5000,n),
                                 absolute ||r||^2 < 1e-5 every 50 iterations,
                                 BiCGSTAB rho0 = 1 + b.b, Richardson w=0.01 x1000) */
    int32_t max_iter;         /* iteration cap (0: 2000) */
    double tol;               /* relative residual ||r||/||b|| target (0: 1e-6) */
    double omega;             /* Richardson weight (0: 0.01) */
    int32_t precond;          /* MPS_PRECOND_* (CG only) */
    int32_t stall_window;     /* FSAI: fall back to Jacobi when the preconditioned
                                 residual r.z has not dropped 4x within this many
                                 iterations (0: 400) */
    int32_t host_loop;        /* 0: the whole iteration loop is one CUDA-graph
                                 launch with a device-side WHILE condition;
                                 1: the host launches the same kernels and polls
                                 the device-side stop flag */
    int32_t reserved;
} mps_solve_opts;

typedef struct {
    int32_t iters;
    int32_t converged;        /* the returned x meets the target: true_resid <= tol
                                 (reference_compat: the reference's stop rule fired) */
    int32_t breakdown;
    int32_t stalled;          /* FSAI-PCG switched to Jacobi */
    int32_t compat_snapshot;  /* reference_compat BiCGSTAB returned its last checkpoint */
    int32_t stop_rule_met;    /* the solver's own stop test on its recurrence residual
                                 fired (the FP32 recurrence can reach tol while the
                                 FP32 x it returns cannot: see true_resid) */
    double rel_resid;         /* recurrence residual ||r||/||b|| at exit */
    double true_resid;        /* ||b - A x|| / ||b|| of the returned x, recomputed on the
                                 GPU after the solve in FP64 (FP64 products and sums
                                 over the stored FP32 matrix and x) */
    int32_t persistent;       /* nonzero: the solve ran as one persistent kernel
                                 (see mps_csr_set_persistent) in its gather (1),
                                 window (2) or stream (3) form; 0: graph form */
    int32_t reserved;
} mps_solve_info;

/* Fill opts with the defaults (tol 1e-6, max_iter 2000, graphs on). */
void mps_solve_opts_default(mps_solve_opts* opts);
const char* mps_last_error_string(void);
const char* mps_status_string(mps_status s);
/* 3: mps_solve_info carries stop_rule_met, true_resid and persistent;
 * 4: persistent (also in mps_ir_info) names the persistent form. */
int32_t mps_abi_version(void);

/* ---- COO -> CSR ------------------------------------------------------- */

/* GPU LSD radix sort of packed (row<<32|col) keys with their values, then the
 * row_ptr count-and-scan.  Bit-exact against a stable sort by key.
 * Replaces csr_tensor::csr_tensor + coo_to_csr_internal
 * (iterative/BiCGSTAB/spmv.cpp:230-268, 62-228). */
mps_status mps_csr_create_from_keys(const uint64_t* d_keys, const float* d_vals, uint64_t nnz,
                                    uint32_t n_rows, uint32_t n_cols, mps_csr** out,
                                    cudaStream_t stream);

/* Wrap an existing CSR (copied into the handle). */
mps_status mps_csr_create_from_csr(const int32_t* d_row_ptr, const int32_t* d_col_ind,
                                   const float* d_vals, uint32_t n_rows, uint32_t n_cols,
                                   uint64_t nnz, mps_csr** out, cudaStream_t stream);

/* Test hook for the bounded device waits (no reference counterpart; the
 * reference's waits are host-side and unbounded): runs the COO -> CSR sort
 * into scratch it frees again, with tile `silent_tile` (tiles of 4096 keys)
 * publishing no look-back status and every look-back wait bounded by
 * `spin_limit` polls, so the tiles after it give up.  Returns MPS_ERR_TIMEOUT
 * (the sort's output is discarded); the device and every handle stay usable. */
mps_status mps_test_sort_lookback_timeout(const uint64_t* d_keys, const float* d_vals, uint64_t nnz,
                                          uint32_t n_rows, uint32_t n_cols, uint32_t spin_limit,
                                          uint32_t silent_tile, cudaStream_t stream);

/* Release a handle (csr_tensor::~csr_tensor, iterative/BiCGSTAB/spmv.cpp:354-366). */
mps_status mps_csr_destroy(mps_csr* A);

mps_status mps_csr_shape(const mps_csr* A, uint32_t* n_rows, uint32_t* n_cols, uint64_t* nnz);

/* Copy the CSR arrays out (the standalone converter's output tensors,
 * spmv_kernel/coo_csr/coo_csr/coo_csr/coo_to_csr.cpp:225-236). */
mps_status mps_csr_export(const mps_csr* A, int32_t* d_row_ptr, int32_t* d_col_ind,
                          float* d_vals, cudaStream_t stream);

/* Standalone converter: sort and write row_ptr/col_ind/out_vals
 * (coo_csr.coo_csr, spmv_kernel/coo_csr/coo_csr/coo_csr/coo_to_csr.cpp:259-288). */
mps_status mps_coo_to_csr(const uint64_t* d_keys, const float* d_vals, uint64_t nnz,
                          uint32_t n_rows, uint32_t n_cols, int32_t* d_row_ptr,
                          int32_t* d_col_ind, float* d_out_vals, cudaStream_t stream);

/* ---- SpMV ------------------------------------------------------------- */

/* y = A x (csr_tensor::mv / mv_internal, iterative/BiCGSTAB/spmv.cpp:421-501;
 * kernel spmv_op, spmv.metal:11-49). */
mps_status mps_csr_spmv(const mps_csr* A, const float* d_x, float* d_y, cudaStream_t stream);

/* SpMV autotuner (no reference counterpart): times the tile-plan candidates
 * (nonzeros per tile: half / default / twice the default; TMA pipeline depth
 * 2 / 3; L2 evict-first hint on the streamed arrays off / on) on this matrix
 * and keeps the fastest for every later SpMV and solve of the handle.  Any
 * pointer may be NULL; h_best_us is the winner's time per SpMV.
 * Synchronises the stream. */
mps_status mps_csr_autotune_spmv(mps_csr* A, int32_t* h_tile_nnz, int32_t* h_stages,
                                 int32_t* h_evict_first, float* h_best_us, cudaStream_t stream);
/* Set the SpMV tile plan by hand (tile_nnz 0: default size, else 256..8192;
 * stages 0: keep, else 2 or 3; evict_first < 0: keep).  No reference
 * counterpart. */
mps_status mps_csr_set_spmv_plan(mps_csr* A, int32_t tile_nnz, int32_t stages,
                                 int32_t evict_first, cudaStream_t stream);

/* y = A x and *d_dot = w . y in FP64 (fused_spvmv, spmv.metal:70-132;
 * deterministic). */
mps_status mps_csr_spmv_dot(const mps_csr* A, const float* d_x, const float* d_w, float* d_y,
                            double* d_dot, cudaStream_t stream);

/* y = A x and *d_dot = w . y for callers that cannot allocate device memory
 * (a process that reserved its whole HBM budget for its own pool at start-up,
 * or a latency-critical path where an allocation, which can synchronise the
 * device, is not allowed).  No counterpart in the reference.
 * Takes the CSR arrays and vectors as device pointers and allocates nothing:
 * its scratch (tile plan, FP64 partial sums, counter) is one file-scope device
 * array of about 280 KB that every GPU loading this library holds until exit.
 * Limit: nnz <= 33,554,432; larger matrices return MPS_ERR_ARG.  d_col_ind and
 * d_vals must be 16-byte aligned (they are read 16 bytes at a time; a
 * cudaMalloc'd buffer is), else MPS_ERR_ARG.  The first call
 * on a device looks up the scratch's device address (cudaGetSymbolAddress), so
 * make that first call before any stream capture.  All calls share the one
 * scratch array: calls that overlap on the GPU (other streams, other threads)
 * race and must not be issued. */
mps_status mps_csr_spmv_dot_noalloc(const int32_t* d_row_ptr, const int32_t* d_col_ind,
                                    const float* d_vals, uint32_t n_rows, uint32_t n_cols,
                                    uint64_t nnz, const float* d_x, const float* d_w, float* d_y,
                                    double* d_dot, cudaStream_t stream);

/* ---- Solvers on CSR --------------------------------------------------- */

/* CG / Jacobi-PCG / learned-FSAI-PCG, x written in place
 * (csr_tensor::cgd / cgd_op, iterative/BiCGSTAB/spmv.cpp:515-659;
 *  iter_solve, iterative/cgd/spmv.cpp:607-747). */
mps_status mps_csr_cg(mps_csr* A, const float* d_b, float* d_x, const mps_solve_opts* opts,
                      mps_solve_info* info, cudaStream_t stream);

/* BiCGSTAB (csr_tensor::bicgstab / bicgstab_op, iterative/BiCGSTAB/spmv.cpp:661-888). */
mps_status mps_csr_bicgstab(mps_csr* A, const float* d_b, float* d_x, const mps_solve_opts* opts,
                            mps_solve_info* info, cudaStream_t stream);

/* Richardson x += w (b - A x) for max_iter iterations
 * (iter_solve / iterative_op, iterative/richardson/spmv.cpp:376-438). */
mps_status mps_csr_richardson(mps_csr* A, const float* d_b, float* d_x,
                              const mps_solve_opts* opts, mps_solve_info* info,
                              cudaStream_t stream);

/* Mixed-precision CG: FP64 outer iterative refinement (residual b - A x and
 * solution in FP64 on the GPU) around FP32 inner CG sweeps whose matrix values
 * are FP32 (value_bits = 32) or BF16 (value_bits = 16).  No reference
 * counterpart (the reference solves in FP32 only). */
typedef struct {
    double tol;               /* outer relative residual target (0: 1e-10) */
    double inner_tol;         /* inner relative reduction per sweep (0: 1e-3 with FP32
                                 values; 0.1 with BF16 values, whose operator differs
                                 from A by about 2^-9 relative, so one sweep cannot
                                 gain much more than that) */
    int32_t max_outer;        /* 0: 50 */
    int32_t max_inner;        /* 0: 2000 */
    int32_t value_bits;       /* 32 or 16 */
    int32_t precond;          /* MPS_PRECOND_NONE / JACOBI / FSAI for the inner CG */
    int32_t host_loop;        /* inner CG iterations launched from the host (see mps_solve_opts) */
    int32_t ir_mode;          /* MPS_IR_AUTO: reliable updates for FP32 values, restarted
                                 refinement for BF16; MPS_IR_RESTART: x += CG(b - A x) sweeps,
                                 each to inner_tol; MPS_IR_REPLACE: one FP32 PCG whose
                                 residual is replaced by the FP64 b - A x each time it has
                                 dropped by inner_tol, with x accumulated in FP64 */
} mps_ir_opts;

enum { MPS_IR_AUTO = 0, MPS_IR_RESTART = 1, MPS_IR_REPLACE = 2 };

typedef struct {
    int32_t outer_iters;      /* refinement sweeps (restart) or residual replacements */
    int32_t inner_iters;      /* total inner CG iterations */
    int32_t converged;
    int32_t persistent;       /* nonzero: the solve ran as one persistent kernel,
                                 1 gather, 2 window, 3 stream form (see
                                 mps_csr_set_persistent) */
    double rel_resid;         /* FP64 true residual at exit */
} mps_ir_info;

/* Reliable-update FSAI-PCG in product form (M = G^T G), plain CG /
 * Jacobi-PCG, BiCGSTAB and Richardson (mps_csr_cg / mps_csr_bicgstab /
 * mps_csr_richardson without reference_compat or host_loop), run as ONE
 * cooperative kernel -- one CTA
 * per SM, grid barriers between the steps of an iteration -- whenever the
 * CTA's share fits its shared memory (about 220 KB): its rows of A (and M)
 * with the vector window they reach (window form), its rows alone (gather
 * form), or -- rows read from L2 in every step -- the window alone (stream
 * form; 2D 5-point systems up to about a million rows).  Otherwise, or
 * with enable = 0, as the CUDA graph of two or three kernels per
 * iteration.  Default 1.  The two compute the same iterates up to the
 * grouping of the FP64 partial sums (Richardson's x: the same bits).  No
 * reference counterpart. */
mps_status mps_csr_set_persistent(mps_csr* A, int32_t enable);

/* Which persistent form the solves above may use: 0 (default) the first
 * that fits -- window, then gather, then stream; 1 gather, 2 window or
 * 3 stream: only that one (the graph form runs when it does not fit).  The
 * forms share the row partition and the per-row arithmetic, so where
 * several fit they return bit-identical results; a choice other than 0 is
 * for comparing them.  No reference counterpart. */
mps_status mps_csr_set_persistent_form(mps_csr* A, int32_t form);

/* Test hook for the persistent kernels' bounded grid-barrier waits (no
 * reference counterpart): runs at most 50 iterations of persistent CG on
 * A with every barrier wait bounded by `spin_limit` polls and CTA
 * `silent_cta` withholding its first arrival (-1: none), so that every
 * CTA's first wait gives up.  Returns MPS_ERR_TIMEOUT (x is then
 * meaningless); the device and the handle stay usable.  MPS_ERR_ARG when
 * the persistent form does not fit A. */
mps_status mps_test_persistent_barrier_timeout(mps_csr* A, const float* d_b, float* d_x, uint32_t spin_limit,
                                               int32_t silent_cta, cudaStream_t stream);

mps_status mps_csr_cg_mixed(mps_csr* A, const double* d_b, double* d_x, const mps_ir_opts* opts,
                            mps_ir_info* info, cudaStream_t stream);

/* ---- Learned FSAI preconditioner ------------------------------------- */

/* Attach a lower-triangular factor G (CSR on tril(A)) so that PCG applies
 * z = G^T (G r).  G's values are copied; its transpose is built on the GPU.
 * No reference counterpart. */
mps_status mps_csr_set_fsai(mps_csr* A, const int32_t* d_g_row_ptr, const int32_t* d_g_col_ind,
                            const float* d_g_vals, uint64_t g_nnz, cudaStream_t stream);

/* How PCG applies the attached factor: SPLIT = two SpMVs (w = G r, z = G^T w),
 * PRODUCT = one SpMV with M = G^T G (built on the GPU from G's pattern, then
 * refreshed from G's values at every attach), AUTO (default) = PRODUCT while
 * M holds at most ~3.75M nonzeros more than G and G^T together (one kernel
 * launch per iteration outweighs the extra bytes), else SPLIT.  The setting
 * applies now to an attached factor and to later ones.  No reference
 * counterpart. */
enum { MPS_FSAI_APPLY_AUTO = 0, MPS_FSAI_APPLY_SPLIT = 1, MPS_FSAI_APPLY_PRODUCT = 2 };
mps_status mps_csr_set_fsai_apply(mps_csr* A, int32_t mode, cudaStream_t stream);
/* The form in force (MPS_FSAI_APPLY_SPLIT / _PRODUCT, -1: no factor) and
 * nnz(M) (0 unless PRODUCT). */
mps_status mps_csr_fsai_apply(const mps_csr* A, int32_t* in_force, uint64_t* nnz_m);
/* Inspection: M = G^T G in CSR (row_ptr n+1, col_ind / values nnz_m), device
 * buffers; PRODUCT form only. */
mps_status mps_csr_fsai_product_get(const mps_csr* A, int32_t* d_row_ptr, int32_t* d_col_ind,
                                    float* d_vals, cudaStream_t stream);

/* Learned FSAI network: per-nonzero MLP 16 -> 64 -> 64 -> 1 (GELU), BF16
 * weights, FP32 accumulation, run on the tensor cores (tcgen05).  It maps 16
 * local coefficient features of each nonzero (i, j) of tril(A) to the factor
 * G (g_ii = softplus(o + log(e-1)) / sqrt(a_ii), g_ij = o / sqrt(a_jj)), so
 * M^-1 = G^T G is SPD.  Parameters: W1[16][64], b1[64], W2[64][64], b2[64],
 * w3[64], b3 (mps_fsai_param_count() floats).  No reference counterpart. */
typedef struct mps_fsai_model mps_fsai_model;
int32_t mps_fsai_param_count(void);
/* h_params NULL: deterministic initialisation close to Jacobi. */
mps_status mps_fsai_model_create(const float* h_params, mps_fsai_model** out);
mps_status mps_fsai_model_destroy(mps_fsai_model* m);
mps_status mps_fsai_model_get(const mps_fsai_model* m, float* h_params);
mps_status mps_fsai_model_set(mps_fsai_model* m, const float* h_params);
/* Build G = net(A) on tril(A) and attach it for MPS_PRECOND_FSAI.  Does
 * not synchronise after the first attach on A (the first one builds the
 * pattern and plans): a bounded tensor-core wait of the network that gave up
 * is reported as MPS_ERR_TIMEOUT by the next solve on A (and by
 * mps_fsai_model_status). */
mps_status mps_fsai_attach(mps_csr* A, const mps_fsai_model* m, cudaStream_t stream);
/* One training step on system A: n_probes Rademacher probes plus n_extra
 * caller vectors (d_extra, n_extra x n, e.g. CG residuals of A); loss
 * L = sum ||v - G A G^T v||^2 / (k n) before the step; Adam with rate lr. */
mps_status mps_fsai_train_step(mps_fsai_model* m, mps_csr* A, int32_t n_probes,
                               const float* d_extra, int32_t n_extra, float lr, uint64_t seed,
                               double* loss, cudaStream_t stream);
/* Inspection: G's pattern and the FP32 features (nnz_g x 16), G's values,
 * raw network passes on FP32 features, and dL/dg for given probes. */
mps_status mps_fsai_features(mps_csr* A, float* d_X, int32_t* d_g_row_ptr, int32_t* d_g_col_ind,
                             uint64_t* nnz_g, cudaStream_t stream);
mps_status mps_fsai_g_values(mps_csr* A, float* d_g_vals, cudaStream_t stream);
mps_status mps_fsai_mlp_forward(const mps_fsai_model* m, const float* d_X, uint64_t N,
                                float* d_out, cudaStream_t stream);
mps_status mps_fsai_mlp_backward(const mps_fsai_model* m, const float* d_X, const float* d_dout,
                                 uint64_t N, float* d_grad, cudaStream_t stream);
mps_status mps_fsai_probe_grad(mps_csr* A, const float* d_V, int32_t k, float* d_grad_g,
                               double* loss, cudaStream_t stream);
/* The same network passes on BF16 features (N x 16, 16-byte aligned), the
 * form attach uses internally: stream-ordered, no allocation and no
 * synchronisation, so they can be chained or timed with events.  A bounded
 * tensor-core wait that gave up is reported by mps_fsai_model_status (which
 * synchronises the stream).  backward_bf16 overwrites d_grad. */
mps_status mps_fsai_mlp_forward_bf16(const mps_fsai_model* m, const void* d_Xbf16, uint64_t N,
                                     float* d_out, cudaStream_t stream);
mps_status mps_fsai_mlp_backward_bf16(const mps_fsai_model* m, const void* d_Xbf16,
                                      const float* d_dout, uint64_t N, float* d_grad,
                                      cudaStream_t stream);
mps_status mps_fsai_model_status(const mps_fsai_model* m, cudaStream_t stream);

/* ---- Batched solve ------------------------------------------------------ */

/* Thousands of independent SPD systems solved by PCG in one persistent,
 * CUDA-graph-captured launch.  The systems are stacked into one block-diagonal
 * CSR (global row and column indices); system s owns rows
 * [h_row_off[s], h_row_off[s+1]).  Groups of warps take systems from a queue
 * ordered largest-first and iterate each to convergence with group-level
 * barriers only.  No reference counterpart. */
typedef struct mps_batch mps_batch;
mps_status mps_batch_create(const int32_t* d_row_ptr, const int32_t* d_col_ind,
                            const float* d_vals, uint64_t nnz, uint32_t total_rows,
                            const int32_t* h_row_off, int32_t n_systems, mps_batch** out,
                            cudaStream_t stream);
mps_status mps_batch_destroy(mps_batch* B);
/* Build the learned factor on the whole block-diagonal matrix. */
mps_status mps_batch_attach_fsai(mps_batch* B, const mps_fsai_model* m, cudaStream_t stream);
/* Per system: MPS_PRECOND_NONE / JACOBI (default) / FSAI, or MPS_BATCH_SKIP
 * (the system is not solved: x untouched, iters 0, converged 0, relres -1). */
#define MPS_BATCH_SKIP 3
mps_status mps_batch_set_precond(mps_batch* B, const int8_t* h_kind);
/* Autotuner: times whole-batch solves with 32, 16, 8, 4, 2, 1 warps per
 * system (stopping once the time grows) and then the cluster path for the
 * largest systems, and keeps the fastest (h_ms: the 6 timings for 1, 2, 4,
 * 8, 16, 32 warps, 0 where not timed; may be NULL).  Overwrites no caller
 * buffer. */
mps_status mps_batch_autotune(mps_batch* B, const float* d_b, double tol, int32_t max_iter,
                              int32_t* h_chosen_wps, float* h_ms, cudaStream_t stream);
int32_t mps_batch_warps_per_system(const mps_batch* B);
/* How many of the batch's largest systems (only systems of 16,384 rows and
 * more qualify) are solved by a thread-block cluster each (chosen by
 * mps_batch_autotune); 0 when the cluster path is off. */
int32_t mps_batch_uses_clusters(const mps_batch* B);
/* Set that number by hand (-1: every qualifying system, 0: off). */
mps_status mps_batch_set_clusters(mps_batch* B, int32_t n_systems);
/* Solve all systems: per-system iteration count, converged flag (the
 * convergence mask) and recurrence relative residual. */
mps_status mps_batch_cg(mps_batch* B, const float* d_b, float* d_x, double tol, int32_t max_iter,
                        int32_t* d_iters, int32_t* d_converged, float* d_relres,
                        cudaStream_t stream);

/* Mixed-precision batched solve: every system's solution accumulated in FP64
 * (d_x64), its Krylov recurrences in FP32, and its residual replaced by the
 * FP64 b - A x (FP64 products over the FP32 matrix) whenever it has dropped
 * by inner_tol since the last replacement (0: 1e-3) or meets tol.  A system
 * stops only when that true residual meets tol; d_relres receives it and
 * d_converged says whether it met tol.  Same launch structure, queue and
 * autotuned warps per system as mps_batch_cg.  No reference counterpart. */
mps_status mps_batch_cg_mixed(mps_batch* B, const float* d_b, double* d_x64, double tol,
                              double inner_tol, int32_t max_iter, int32_t* d_iters,
                              int32_t* d_converged, float* d_relres, cudaStream_t stream);

/* ---- BCSR --------------------------------------------------------------- */

/* BCSR from pre-built block arrays: row-major B x B blocks (B = 4 or 8),
 * block row_ptr/col_ind; n_rows/n_cols are the logical sizes, padded up to a
 * multiple of B (bcsr_tensor::bcsr_tensor, iterative/BiCGSTAB/bcsr.cpp:357-422). */
mps_status mps_bcsr_create(const float* d_vals, const int32_t* d_row_ptr,
                           const int32_t* d_col_ind, uint64_t n_blocks, uint32_t n_rows,
                           uint32_t n_cols, uint32_t block, mps_bcsr** out,
                           cudaStream_t stream);

/* BCSR built on the GPU from packed COO keys: radix sort on block keys, then
 * block densification (replaces the scipy path coo_to_metal_bcsr,
 * iterative/BiCGSTAB/bcsr_benchmark.py:36-66). */
mps_status mps_bcsr_create_from_keys(const uint64_t* d_keys, const float* d_vals, uint64_t nnz,
                                     uint32_t n_rows, uint32_t n_cols, uint32_t block,
                                     mps_bcsr** out, cudaStream_t stream);

mps_status mps_bcsr_destroy(mps_bcsr* A);
mps_status mps_bcsr_shape(const mps_bcsr* A, uint32_t* n_block_rows, uint64_t* n_blocks,
                          uint32_t* block, uint32_t* padded_n);
mps_status mps_bcsr_export(const mps_bcsr* A, int32_t* d_row_ptr, int32_t* d_col_ind,
                           float* d_vals, cudaStream_t stream);

/* y = A x on padded vectors (spmv_op, iterative/BiCGSTAB/bcsr_spmv.metal:30-69). */
mps_status mps_bcsr_spmv(const mps_bcsr* A, const float* d_x, float* d_y, cudaStream_t stream);

/* CG and BiCGSTAB on BCSR; b and x are padded vectors
 * (bcsr_tensor::cgd_op / bicgstab_op, iterative/BiCGSTAB/bcsr.cpp:590-721, 761-949). */
mps_status mps_bcsr_cg(mps_bcsr* A, const float* d_b, float* d_x, const mps_solve_opts* opts,
                       mps_solve_info* info, cudaStream_t stream);
mps_status mps_bcsr_bicgstab(mps_bcsr* A, const float* d_b, float* d_x,
                             const mps_solve_opts* opts, mps_solve_info* info,
                             cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* MPSPARSE_H */
