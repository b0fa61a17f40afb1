// internal.hpp -- host-side structures shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/mpsparse.h"

namespace mps {

// ---- error plumbing -------------------------------------------------------
void set_error(const std::string& msg);
mps_status fail(mps_status s, const std::string& msg);
mps_status cuda_fail(cudaError_t e, const char* what);
#define MPS_CUDA(call)                                             \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) return ::mps::cuda_fail(_e, #call); \
    } while (0)

int num_sms();
size_t l2_bytes();        // L2 cache of the current device

// Stream-ordered scratch allocations of the library come from one memory
// pool per device that keeps its memory after frees (release threshold at
// the maximum): a large sort's temporary buffers are mapped once, not on
// every call.  The pool holds at most the library's peak scratch footprint.
cudaMemPool_t lib_pool();
template <class T>
inline cudaError_t stream_alloc(T** p, size_t bytes, cudaStream_t s) {
    cudaMemPool_t pool = lib_pool();
    if (!pool) return cudaErrorMemoryAllocation;
    return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, pool, s);
}

// Long-lived buffers of handles (matrix arrays, tile plans, solver and
// factor work areas) come from the same pool: a fresh handle then costs no
// driver allocation, and destroying one returns its memory to the pool
// instead of unmapping it.  Allocated on the stream of the call that creates
// the buffer (ordered before its first use there); dev_free synchronises the
// device first, as cudaFree does, so no kernel on any stream still reads
// the buffer when it goes back to the pool.
template <class T>
inline cudaError_t dev_alloc(T** p, size_t bytes, cudaStream_t s) {
    return stream_alloc(p, bytes ? bytes : 16, s);
}
inline void dev_free(void* p) {
    if (!p) return;
    cudaDeviceSynchronize();
    cudaFreeAsync(p, cudaStreamLegacy);
}

// Pinned host blocks (the solvers' scalar mirrors) and non-blocking capture
// streams are kept per process / per device and handed to the next handle:
// pinning host memory and creating streams cost far more than a solve's
// other set-up.
void* pinned_block_get(size_t bytes);    // up to 4 KB, zeroed
void pinned_block_put(void* p);
cudaStream_t capture_stream_get();       // on the current device
void capture_stream_put(cudaStream_t s);

// ---- device scalar block of one solve --------------------------------------
// One instance lives in device memory per handle; the host mirrors it into
// pinned memory at the end of a solve.
struct DevScalars {
    // Krylov scalars (FP64: the alpha/beta/omega reductions run in FP64)
    double rr, rz, pq, alpha, beta;
    double rho, rho_old, omega, sigma, phi1, phi2, rnorm2;
    double bnorm2, tol2, staged, best_rr;
    double omega_rich;
    double rz_jac;      // r . D^-1 r of the last update (Jacobi fallback)
    double true_rr;     // ||b - A x||^2 of the returned x in FP64 (after the solve)
    // control
    int iter, max_iter, done, converged, breakdown, stalled, snapshot, compat;
    int mode;           // preconditioner in force: 0 none, 1 Jacobi, 2 FSAI
    int best_iter, stall_window, err;
    int n;              // rows
    int restart;        // next direction update restarts (beta = 0)
    int guard;          // loop bodies executed (watchdog)
    int guard_limit;    // watchdog bound: a loop never runs more bodies than this
    // reliable updates (mixed-precision CG): FP64 solution, residual replacement
    double rr_ref;      // largest recurrence ||r||^2 since the last replacement
    double delta2;      // replace when ||r||^2 < delta2 * rr_ref (or at the target)
    int replace;        // a replacement is due in this iteration
    int replaced;       // replacements so far
    int refresh;        // FSAI: the replaced residual still needs its G-apply
};

// Parameters copied host->device before each solve.
struct SolveParams {
    double tol;
    double omega;
    int max_iter;
    int compat;
    int precond;
    int stall_window;
    double delta;       // reliable updates: residual drop between replacements
};

// ---- CSR views ---------------------------------------------------------------
struct CsrDev {
    const int* rp;
    const int* ci;
    const float* v;
    const __nv_bfloat16* vb;
    const int* tile_row;   // ntiles + 1 row boundaries of the SpMV tiles
    int n_rows;
    int ntiles;
    int cap;               // shared-memory product capacity of a tile
};

struct SpmvPlan {
    int tile_nnz = 0;      // target nnz per tile
    int ntiles = 0;
    int cap = 0;
    int grid = 0;          // persistent CTAs
    int* d_tile_row = nullptr;
    int4* d_meta = nullptr;   // per tile {row begin, row end, nnz begin, nnz end}
    int cap_s = 0;            // staged nonzeros per buffer of the TMA kernel
    int rcap = 0;             // staged row_ptr entries per buffer
    int grid_s = 0;           // persistent CTAs of the TMA kernel
    int stages = 2;           // TMA pipeline depth (2 or 3)
    int evict_first = 1;      // L2 evict-first hint on the col_ind/value copies
    bool evict_auto = true;   // hint chosen by size (no caller set it)
    int max_tile_nnz = 0;     // largest tile (nonzeros) and row count of the plan
    int max_tile_rows = 0;
};

// View of a CSR for the TMA-staged kernel (csr_stream.cuh).
struct CsrStreamDev {
    const int* rp;
    const int* ci;
    const float* v;
    const __nv_bfloat16* vb;
    const int4* meta;
    int ntiles;
    int cap;
    int rcap;
    int evict_first;
    unsigned* err;
};

// Launch geometry of the streaming vector kernels.
struct VecGeom {
    int grid;
    int n4;                // float4 count over the padded length
};

constexpr int kNT = 256;           // threads per CTA of the solver kernels
constexpr int kMaxPartials = 4096; // FP64 partial slots per reduction
constexpr int kMaxDevices = 64;    // per-device host caches (device ordinals below this)
constexpr int kMinTileNnz = 512;   // smallest default SpMV tile (nonzeros); sizes static tile plans

// Solver workspace owned by a handle (lazily allocated, padded to x4 floats).
struct Workspace {
    size_t n_pad = 0;
    float* vec[12] = {};
    double* partials = nullptr;    // 4 * kMaxPartials
    unsigned* counters = nullptr;  // 16
    DevScalars* sc = nullptr;
    DevScalars* h_sc = nullptr;    // pinned mirror
    SolveParams* d_params = nullptr;
};

struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
};

struct CsrMat {
    int32_t* rp = nullptr;
    int32_t* ci = nullptr;
    float* v = nullptr;
    uint32_t n_rows = 0, n_cols = 0;
    uint64_t nnz = 0;
    SpmvPlan plan;
    unsigned* err = nullptr;   // device error word (bounded-wait timeouts)
    CsrDev view(const __nv_bfloat16* vb = nullptr) const {
        return CsrDev{rp, ci, v, vb, plan.d_tile_row, (int)n_rows, plan.ntiles, plan.cap};
    }
    CsrStreamDev stream_view(const __nv_bfloat16* vb = nullptr) const {
        return CsrStreamDev{rp, ci, v, vb, plan.d_meta, plan.ntiles, plan.cap_s, plan.rcap,
                            plan.evict_first, err};
    }
};

// Spare elements after each CSR array: 16-byte-rounded bulk copies of a tile
// never leave the allocation.
constexpr int kCsrPad = 16;

// ---- internal entry points ---------------------------------------------------
// Sort packed keys into CSR arrays (caller-allocated outputs).  `payload` is
// moved as 32-bit words.  Returns a CUDA error; device-side range / timeout
// errors are OR-ed into *d_err.  spin_limit (0: the standard bound) and
// silent_tile (a tile that publishes no look-back status; none by default)
// exist for the bounded-wait test hook only.
cudaError_t sort_to_csr(const uint64_t* keys, const uint32_t* payload, uint64_t nnz,
                        uint32_t n_rows, uint32_t n_cols, int32_t* row_ptr, int32_t* col_out,
                        uint32_t* payload_out, unsigned* d_err, cudaStream_t s,
                        unsigned spin_limit = 0, unsigned silent_tile = 0xffffffffu);

// Tile plan of A (tile_nnz <= 0: the default size; stages <= 0 /
// evict_first < 0: keep the current plan's choice).  Synchronises `s` once to
// size the staging buffers to the largest tile.
cudaError_t spmv_plan_build(CsrMat& A, int tile_nnz, cudaStream_t s, int stages = 0,
                            int evict_first = -1);
void spmv_plan_free(SpmvPlan& p);
cudaError_t spmv_launch(const CsrMat& A, const float* x, float* y, cudaStream_t s);
cudaError_t spmv_dot_launch(const CsrMat& A, const float* x, const float* w, float* y,
                            double* d_dot, double* partials, unsigned* counter,
                            cudaStream_t s);

}  // namespace mps
