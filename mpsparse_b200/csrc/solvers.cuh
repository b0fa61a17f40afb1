// solvers.cuh -- Krylov solvers with every iteration on the device.
//
// The reference drives CG / BiCGSTAB / Richardson from the host with 3-6
// kernel dispatches per iteration, relaxed float atomics for the dots and a
// host round-trip every 50 iterations (iterative/BiCGSTAB/spmv.cpp:528-888,
// iterative/richardson/spmv.cpp:376-425).  Here:
//   * each dot product is fused into the kernel that produces its operand
//     (SpMV epilogue or axpy) and reduced deterministically in FP64: per-CTA
//     partials, then the last CTA sums them in a fixed order and updates the
//     FP64 scalars (alpha, beta, omega, rho) in device memory;
//   * stop rules run on the device: the last CTA of the last kernel of an
//     iteration writes the CUDA-graph WHILE condition, so a whole solve is one
//     graph launch with no host synchronisation until the end;
//   * every kernel of an iteration returns immediately once the stop flag is
//     set, so a solve never overshoots its result.
#pragma once
#include "spmv_kernels.cuh"

namespace mps {

struct Ctx {
    DevScalars* sc;
    double* part;          // 4 * kMaxPartials doubles
    unsigned* ctr;         // 16 counters
    cudaGraphConditionalHandle h;     // WHILE condition of the solve loop
    int use_cond;
    cudaGraphConditionalHandle hif;   // IF condition of the replacement branch
};

__device__ __forceinline__ void set_cond(const Ctx& c, bool run) {
    if (c.use_cond) cudaGraphSetConditional(c.h, run ? 1u : 0u);
}

// Two-sum block reduction + last-CTA election, shared by the vector kernels.
template <int NS>
__device__ __forceinline__ bool reduce_partials(const Ctx& c, int slot, const double* acc,
                                                double* tot) {
    __shared__ double red[NS * (kNT / 32)];
    __shared__ int last_flag;
    double v[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) v[i] = acc[i];
    block_sum_n<kNT, NS>(v, red);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NS; ++i) c.part[i * kMaxPartials + blockIdx.x] = v[i];
    }
    if (!arrive_last(c.ctr + slot, &last_flag)) return false;
    double t[NS];
    sum_partials_n<kNT, NS>(c.part, kMaxPartials, gridDim.x, red, t);
#pragma unroll
    for (int i = 0; i < NS; ++i) tot[i] = t[i];
    return true;
}

__device__ __forceinline__ double dot4(float4 a, float4 b) {
    return (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
}
__device__ __forceinline__ double dot4w(float4 a, float4 w) {   // sum a^2 * w
    return (double)a.x * a.x * w.x + (double)a.y * a.y * w.y + (double)a.z * a.z * w.z +
           (double)a.w * a.w * w.w;
}
__device__ __forceinline__ float4 axpy4(float a, float4 x, float4 y) {   // y + a x
    return make_float4(fmaf(a, x.x, y.x), fmaf(a, x.y, y.y), fmaf(a, x.z, y.z), fmaf(a, x.w, y.w));
}
__device__ __forceinline__ float4 mul4(float4 a, float4 b) {
    return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w);
}

// Watchdog of a device-side loop, run by one thread of the last kernel of each
// loop body: stops the loop (and flags a timeout) once it has executed more
// bodies than the iteration cap allows, whatever happened to the reductions.
__device__ __forceinline__ void loop_watchdog(DevScalars* s) {
    if (++s->guard > s->guard_limit) {
        s->done = 1;
        s->err |= kErrTimeout;
    }
}

#define MPS_GRID_STRIDE(i, n) \
    for (int i = blockIdx.x * kNT + threadIdx.x; i < (n); i += gridDim.x * kNT)

// ============================ CG / PCG =====================================
// Counter slots: 0 init, 1 pq, 2 xr, 3 G-apply, 4..7 BiCGSTAB, 8 Richardson.

static __device__ void cg_init_scalars(const Ctx& c, const SolveParams* __restrict__ prm, int n,
                                       int mode, double bb, double bzb);

// x = 0, r = b, p = M b; rr = b.b, rz = b.Mb; stop flags reset.
static __global__ void __launch_bounds__(kNT)
cg_init(const float4* __restrict__ b, float4* __restrict__ x, float4* __restrict__ r,
        float4* __restrict__ p, const float4* __restrict__ dinv, int n4, int n,
        const SolveParams* __restrict__ prm, Ctx c) {
    pdl_begin();
    const int mode = prm->precond;
    double acc[2] = {0.0, 0.0};
    MPS_GRID_STRIDE(i, n4) {
        const float4 bv = b[i];
        x[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        r[i] = bv;
        float4 z = bv;
        if (mode == 1) {
            const float4 d = dinv[i];
            z = mul4(bv, d);
            acc[1] += dot4w(bv, d);
        }
        if (mode != 2) p[i] = z;
        acc[0] += dot4(bv, bv);
    }
    double tot[2];
    if (!reduce_partials<2>(c, 0, acc, tot)) return;
    if (threadIdx.x != 0) return;
    cg_init_scalars(c, prm, n, mode, tot[0], tot[1]);
}

// Scalars of a CG / PCG start: ||b||^2 = bb, b.D^-1 b = bzb.
static __device__ void cg_init_scalars(const Ctx& c, const SolveParams* __restrict__ prm, int n,
                                       int mode, double bb, double bzb) {
    DevScalars* s = c.sc;
    s->n = n;
    s->compat = prm->compat;
    s->max_iter = prm->compat ? (n < 1000 ? n : 1000) : prm->max_iter;
    s->iter = 0;
    s->done = 0;
    s->converged = 0;
    s->breakdown = 0;
    s->stalled = 0;
    s->snapshot = 0;
    s->err = 0;
    s->mode = prm->compat ? 0 : mode;
    s->stall_window = prm->stall_window;
    s->restart = (mode == 2) ? 1 : 0;   // the first G-apply starts the direction
    s->bnorm2 = bb;
    s->rr = bb;
    s->rz = (mode == 1) ? bzb : bb;
    s->tol2 = prm->tol * prm->tol * bb;
    s->best_rr = 1e300;
    s->best_iter = 0;
    s->beta = 0.0;
    s->rz_jac = 0.0;
    s->guard = 0;
    s->guard_limit = s->max_iter + 8;
    s->rr_ref = bb;
    s->delta2 = prm->delta * prm->delta;
    s->replace = 0;
    s->replaced = 0;
    s->refresh = 0;
    if (!isfinite(bb)) {
        s->err = kErrNotFinite;
        s->done = 1;
    } else if (!prm->compat && bb == 0.0) {
        s->done = 1;
        s->converged = 1;
    } else if (s->max_iter <= 0) {
        s->done = 1;
    }
    set_cond(c, !s->done);
}

// q = A p ; pq = p.q ; alpha = rz / pq
struct EpiCgPq {
    static constexpr bool kPre = true;   // solver loops only
    static constexpr int NS = 1;
    float* q;
    const float* p;
    DevScalars* sc;
    unsigned* counter;
    double* partials;
    __device__ bool active() const { return !sc->done; }
    __device__ void tick() const {}
    __device__ void on_skip() const {}
    __device__ void row(int r, float s, double* acc) const {
        q[r] = s;
        acc[0] += (double)p[r] * (double)s;
    }
    __device__ void finalize(const double* tot) const {
        const double pq = tot[0];
        sc->pq = pq;
        double alpha;
        if (sc->compat) {                                    // cgd.metal:38-42
            alpha = fabs(pq) > 1e-9 ? sc->rz / pq : 0.0;
        } else if (!(pq > 0.0) || !isfinite(pq)) {
            sc->breakdown = 1;
            sc->done = 1;
            alpha = 0.0;
        } else {
            alpha = sc->rz / pq;
        }
        sc->alpha = alpha;
    }
};

// beta and rz of the next direction (no preconditioner / Jacobi; the FSAI
// step sets them from w.w itself).
static __device__ void cg_direction(DevScalars* s, double rr_new, double rz_jac) {
    s->rz_jac = rz_jac;
    if (s->mode == 1) {
        s->beta = s->restart ? 0.0 : rz_jac / s->rz;
        s->rz = rz_jac;
        s->restart = 0;
    } else if (s->mode == 0) {
        s->beta = rr_new / s->rz;
        s->rz = rr_new;
    }
}

static __device__ void cg_finalize_xr(DevScalars* s, double rr_new, double rz_jac) {
    const int it = ++s->iter;
    const double rr_old = s->rr;
    s->rr = rr_new;
    if (s->compat) {
        // spmv.cpp:603-627: every 50 iterations, on the value before this update
        if ((it - 1) % 50 == 0 && rr_old < 1e-5) {
            s->done = 1;
            s->converged = 1;
        } else if (it >= s->max_iter) {
            s->done = 1;
        }
        s->beta = rr_new / rr_old;                           // cgd.metal:81, unguarded
        s->rz = rr_new;
        return;
    }
    if (!isfinite(rr_new)) {
        s->breakdown = 1;
        s->done = 1;
        return;
    }
    if (rr_new <= s->tol2) {
        s->converged = 1;
        s->done = 1;
        return;
    }
    if (it >= s->max_iter) {
        s->done = 1;
        return;
    }
    cg_direction(s, rr_new, rz_jac);
}

// x += alpha p ; r -= alpha q ; rr = r.r (and r.D^-1 r when a diagonal exists)
static __global__ void __launch_bounds__(kNT)
cg_update_xr(float4* __restrict__ x, float4* __restrict__ r, const float4* __restrict__ p,
             const float4* __restrict__ q, const float4* __restrict__ dinv, int n4, Ctx c) {
    pdl_begin();
    if (c.sc->done) return;
    const float a = (float)c.sc->alpha;
    double acc[2] = {0.0, 0.0};
    MPS_GRID_STRIDE(i, n4) {
        const float4 pv = p[i], qv = q[i];
        x[i] = axpy4(a, pv, x[i]);
        const float4 rv = axpy4(-a, qv, r[i]);
        r[i] = rv;
        acc[0] += dot4(rv, rv);
        if (dinv) acc[1] += dot4w(rv, dinv[i]);
    }
    double tot[2];
    if (!reduce_partials<2>(c, 2, acc, tot)) return;
    if (threadIdx.x == 0) cg_finalize_xr(c.sc, tot[0], tot[1]);
}

// ---- reliable updates (mixed-precision CG) ----------------------------------
// The FP32 recurrences run as above; x is accumulated in FP64, and whenever
// the recurrence residual has dropped by delta since the last replacement (or
// reaches the target) r is replaced by the FP64 true residual b - A x
// (Sleijpen & van der Vorst's reliable updates).  The solve stops only on a
// replaced, i.e. true, residual.

// x = 0 (FP64), r = (float)b, p = M r; bb = ||b||^2 in FP64.
static __global__ void __launch_bounds__(kNT)
cg_init_ir(const double* __restrict__ b, double* __restrict__ x, float* __restrict__ r,
           float* __restrict__ p, const float* __restrict__ dinv, int n,
           const SolveParams* __restrict__ prm, Ctx c) {
    pdl_begin();
    const int mode = prm->precond;
    double acc[2] = {0.0, 0.0};
    MPS_GRID_STRIDE(i, n) {
        const double bd = b[i];
        const float bf = (float)bd;
        x[i] = 0.0;
        r[i] = bf;
        float z = bf;
        if (mode == 1) {
            z = bf * dinv[i];
            acc[1] += (double)bf * bf * dinv[i];
        }
        if (mode != 2) p[i] = z;
        acc[0] += bd * bd;
    }
    double tot[2];
    if (!reduce_partials<2>(c, 0, acc, tot)) return;
    if (threadIdx.x != 0) return;
    cg_init_scalars(c, prm, n, mode, tot[0], tot[1]);
}

static __device__ void cg_finalize_ir(DevScalars* s, double rr_new, double rz_jac) {
    const int it = ++s->iter;
    s->rr = rr_new;
    if (!isfinite(rr_new)) {
        s->breakdown = 1;
        s->done = 1;
        return;
    }
    if (rr_new > s->rr_ref) s->rr_ref = rr_new;
    if (rr_new <= s->tol2 || rr_new < s->delta2 * s->rr_ref) {
        s->replace = 1;                  // the replacement step sets the direction
        s->rz_jac = rz_jac;
        return;
    }
    if (it >= s->max_iter) {
        s->done = 1;
        return;
    }
    cg_direction(s, rr_new, rz_jac);
}

// x += alpha p (FP64) ; r -= alpha q ; rr = r.r, r.D^-1 r
static __global__ void __launch_bounds__(kNT)
cg_update_xr_ir(double* __restrict__ x, float* __restrict__ r, const float* __restrict__ p,
                const float* __restrict__ q, const float* __restrict__ dinv, int n, Ctx c) {
    pdl_begin();
    if (c.sc->done) return;
    const double a = c.sc->alpha;
    const float af = (float)a;
    double acc[2] = {0.0, 0.0};
    MPS_GRID_STRIDE(i, n) {
        const float pv = p[i];
        x[i] = fma(a, (double)pv, x[i]);
        const float rv = fmaf(-af, q[i], r[i]);
        r[i] = rv;
        acc[0] += (double)rv * rv;
        if (dinv) acc[1] += (double)rv * rv * dinv[i];
    }
    double tot[2];
    if (!reduce_partials<2>(c, 2, acc, tot)) return;
    if (threadIdx.x == 0) cg_finalize_ir(c.sc, tot[0], tot[1]);
}

// Replacement (runs only when due): r = (float)(b - A x) with FP64 gathers of
// x and FP64 sums; ||b - A x||^2 and r.D^-1 r; then the stop test and the
// next direction.
// With FSAI the residual is a pair of buffers (r, r1; the current one is
// picked by iteration parity) and the replaced residual is flagged for its
// G-apply (EpiFsai1R).
struct EpiReplace {
    static constexpr int NS = 2;
    const double* b;
    float* r;
    const float* dinv;
    DevScalars* sc;
    unsigned* counter;
    double* partials;
    float* r1 = nullptr;
    Ctx c = {};                    // loop: c.h is the condition of the loop
    int loop = 0;                  //   around the iterations and this step
    float* rw = nullptr;           // per thread: the buffer written
    __device__ bool active() const { return !sc->done && sc->replace; }
    __device__ void tick() const {
        if (loop) set_cond(c, !sc->done);
    }
    __device__ void on_skip() const {}
    __device__ void begin() { rw = (r1 && (sc->iter & 1)) ? r1 : r; }
    __device__ void row(int i, double s, double* acc) const {
        const double rt = b[i] - s;
        const float rf = (float)rt;
        rw[i] = rf;
        acc[0] += rt * rt;
        acc[1] += (double)rf * rf * (dinv ? dinv[i] : 1.f);
    }
    __device__ void finalize(const double* tot) const {
        DevScalars* s = sc;
        s->replace = 0;
        ++s->replaced;
        const double rr = tot[0];
        s->rr = rr;
        s->rr_ref = rr;
        if (!isfinite(rr)) {
            s->breakdown = 1;
            s->done = 1;
        } else if (rr <= s->tol2) {
            s->converged = 1;
            s->done = 1;
        } else if (s->iter >= s->max_iter) {
            s->done = 1;
        } else {
            cg_direction(s, rr, tot[1]);
            if (r1 && s->mode == 2) s->refresh = 1;
        }
        if (loop) set_cond(c, !s->done);
    }
};

// p = z + beta p with z = r (no preconditioner) or D^-1 r (Jacobi).  Last
// kernel of a CG iteration: writes the WHILE condition.
static __global__ void __launch_bounds__(kNT)
cg_update_p(float4* __restrict__ p, const float4* __restrict__ r, const float4* __restrict__ dinv,
            int n4, Ctx c) {
    pdl_begin();
    DevScalars* s = c.sc;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        loop_watchdog(s);
        set_cond(c, !s->done);
    }
    if (s->done || s->mode == 2) return;
    const float beta = (float)s->beta;
    const bool jac = s->mode == 1;
    MPS_GRID_STRIDE(i, n4) {
        float4 z = r[i];
        if (jac) z = mul4(z, dinv[i]);
        p[i] = axpy4(beta, p[i], z);
    }
}

// beta = rz / rz_old of an FSAI direction, rz = r.G^T G r = ||G r||^2.
// Stall watch on rz: when it has not dropped 4x within stall_window
// iterations, fall back to Jacobi (restart the direction from z = D^-1 r).
static __device__ void fsai_beta(DevScalars* sc, double rz) {
    const int it = sc->iter;
    if (!sc->restart && sc->stall_window > 0) {
        if (rz < 0.25 * sc->best_rr) {
            sc->best_rr = rz;
            sc->best_iter = it;
        } else if (it - sc->best_iter >= sc->stall_window) {
            sc->mode = 1;
            sc->stalled = 1;
            sc->beta = 0.0;
            sc->rz = sc->rz_jac;
            sc->restart = 0;
            return;
        }
    }
    sc->beta = sc->restart ? 0.0 : rz / sc->rz;
    sc->rz = rz;
    sc->restart = 0;
}

// FSAI step 1: w = G r ; rz = w.w (= r.G^T G r) ; beta = rz / rz_old
struct EpiFsai1 {
    static constexpr bool kPre = true;   // solver loops only
    static constexpr int NS = 1;
    float* w;
    DevScalars* sc;
    unsigned* counter;
    double* partials;
    __device__ bool active() const { return !sc->done && sc->mode == 2; }
    __device__ void tick() const {}
    __device__ void on_skip() const {}
    __device__ void row(int r, float s, double* acc) const {
        w[r] = s;
        acc[0] += (double)s * (double)s;
    }
    __device__ void finalize(const double* tot) const { fsai_beta(sc, tot[0]); }
};

// The G-apply of a replaced residual (reliable updates): w = G r with r the
// current buffer of the pair; runs only after a replacement.
struct EpiFsai1R : EpiFsai1 {
    const float* r0 = nullptr;
    const float* r1 = nullptr;
    const float* rc = nullptr;     // per thread: the current buffer
    __device__ bool active() const { return !sc->done && sc->mode == 2 && sc->refresh; }
    __device__ void begin() { rc = (sc->iter & 1) ? r1 : r0; }
    __device__ float gather(int c) const { return __ldg(rc + c); }
    __device__ void finalize(const double* tot) const {
        sc->refresh = 0;
        fsai_beta(sc, tot[0]);
    }
};

// Fused FSAI-PCG step (one kernel in place of the x/r update and the G-apply):
//   r' = r - alpha q          (FP32, the same fmaf as the unfused update)
//   x += alpha p              (FP64 under reliable updates, else FP32)
//   w = G r'                  with r' gathered as r[c] - alpha q[c]
//   sums r'.r', r'.D^-1 r', w.w
// r' goes to the other buffer of the residual pair (the current one is
// r[iter & 1]), so no CTA overwrites an element another CTA still gathers.
// The last CTA advances the iteration and, under reliable updates, decides
// whether a replacement is due (then the IF branch of the graph runs
// EpiReplace and EpiFsai1R); otherwise it sets the next direction's beta.
template <bool IR>
struct EpiFsaiR {
    static constexpr bool kPre = true;   // solver loops only
    static constexpr int NS = 3;
    const float* r0;
    const float* r1;
    const float* q;
    const float* p;
    std::conditional_t<IR, double, float>* x;
    const float* dinv;             // null: no diagonal
    float* w;
    DevScalars* sc;
    unsigned* counter;
    double* partials;
    Ctx c;
    const float* rc = nullptr;     // per thread (begin): current residual
    float* rn = nullptr;           //   the buffer r' goes to
    double a = 0.0;
    float af = 0.f;
    __device__ bool active() const { return !sc->done; }
    __device__ void tick() const {}
    __device__ void on_skip() const {}
    __device__ void begin() {
        const bool odd = sc->iter & 1;
        rc = odd ? r1 : r0;
        rn = const_cast<float*>(odd ? r0 : r1);
        a = sc->alpha;
        af = (float)a;
    }
    __device__ float gather(int col) const { return fmaf(-af, __ldg(q + col), __ldg(rc + col)); }
    __device__ void row(int i, float s, double* acc) const {
        const float rv = fmaf(-af, q[i], rc[i]);
        rn[i] = rv;
        if constexpr (IR) x[i] = fma(a, (double)p[i], x[i]);
        else x[i] = fmaf(af, p[i], x[i]);
        w[i] = s;
        acc[0] += (double)rv * rv;
        if (dinv) acc[1] += (double)rv * rv * dinv[i];
        acc[2] += (double)s * (double)s;
    }
    __device__ void finalize(const double* tot) const {
        DevScalars* s = sc;
        if constexpr (IR) {
            cg_finalize_ir(s, tot[0], tot[1]);
            if (c.use_cond) cudaGraphSetConditional(c.hif, s->replace ? 1u : 0u);
            if (s->replace || s->done) return;
        } else {
            cg_finalize_xr(s, tot[0], tot[1]);
            if (s->done) return;
        }
        if (s->mode == 2) fsai_beta(s, tot[2]);
    }
};

// FSAI step 2: p = G^T w + beta p
// As the last kernel of an FSAI-PCG iteration (`body`) it also takes
// cg_update_p's place: it runs the loop watchdog and writes the WHILE
// condition at its start (the stop decision is final by then), and after a
// stall fallback it updates p = D^-1 r + beta p instead (the G^T w row sum is
// then unused).
struct EpiFsai2 {
    static constexpr bool kPre = true;   // solver loops only
    static constexpr int NS = 0;
    float* p;
    DevScalars* sc;
    unsigned* counter = nullptr;
    double* partials = nullptr;
    const float* r = nullptr;      // body only: the residual pair (r, r1)
    const float* dinv = nullptr;
    Ctx c = {};
    int body = 0;
    const float* r1 = nullptr;
    const float* rc = nullptr;     // per thread: the current residual
    __device__ bool active() const { return !sc->done && (body ? sc->mode >= 1 : sc->mode == 2); }
    __device__ void begin() { rc = (r1 && (sc->iter & 1)) ? r1 : r; }
    __device__ void tick() const {
        if (body) {
            loop_watchdog(sc);
            set_cond(c, !sc->done);
        }
    }
    __device__ void on_skip() const {}
    __device__ void row(int i, float s, double*) const {
        const float beta = (float)__ldcg(&sc->beta);
        if (!body || __ldcg(&sc->mode) == 2) {
            p[i] = fmaf(beta, p[i], s);
        } else {
            const float z = rc[i] * dinv[i];
            p[i] = beta != 0.f ? fmaf(beta, p[i], z) : z;
        }
    }
    __device__ void finalize(const double*) const {}
};

// ---- FSAI-PCG with M = G^T G (one SpMV per preconditioner apply) ------------
// Two kernels per iteration:
//   K1  p_k = z + beta p_(k-1) formed on the fly (gathered, and written to
//       p[k & 1] for the own rows), q = A p_k, p.q -> alpha      (EpiCgPqZ)
//   K2  r' = r - alpha q, x += alpha p_k, z = M r' (r' gathered on the fly,
//       written to the other buffer of the residual pair), r'.r', r'.D^-1 r',
//       r'.z -> replacement decision or beta, loop condition      (EpiFsaiM)
// After a Jacobi fallback (stall), K1 forms z = D^-1 r itself.  Under
// reliable updates the graph nests two loops: the inner one runs iterations
// (several per body) until a replacement is due or the solve stops; the
// outer one then runs the replacement (EpiReplace) and z = M r (EpiMzR),
// which set the outer condition and re-arm the inner one.

// z = M r (init) ; rz = r.z ; beta (restarts the direction)
struct EpiMz {
    static constexpr bool kPre = true;   // solver loops only
    static constexpr int NS = 1;
    float* z;
    DevScalars* sc;
    unsigned* counter;
    double* partials;
    const float* r;                // residual M is applied to (own rows, for r.z)
    __device__ bool active() const { return !sc->done && sc->mode == 2; }
    __device__ void tick() const {}
    __device__ void on_skip() const {}
    __device__ void row(int i, float s, double* acc) const {
        z[i] = s;
        acc[0] += (double)r[i] * (double)s;
    }
    __device__ void finalize(const double* tot) const { fsai_beta(sc, tot[0]); }
};

// z = M r for a replaced residual (current buffer of the pair); after a
// replacement only.
struct EpiMzR {
    static constexpr bool kPre = true;   // solver loops only
    static constexpr int NS = 1;
    float* z;
    DevScalars* sc;
    unsigned* counter;
    double* partials;
    const float* r0;
    const float* r1;
    Ctx c = {};                    // loop: c.h is the iterations' loop, re-armed
    int loop = 0;                  //   for the next round
    const float* rc = nullptr;     // per thread: current residual
    __device__ bool active() const { return !sc->done && sc->mode == 2 && sc->refresh; }
    __device__ void tick() const {
        if (loop) set_cond(c, !sc->done);
    }
    __device__ void on_skip() const {}
    __device__ void begin() { rc = (sc->iter & 1) ? r1 : r0; }
    __device__ float gather(int c) const { return __ldg(rc + c); }
    __device__ void row(int i, float s, double* acc) const {
        z[i] = s;
        acc[0] += (double)rc[i] * (double)s;
    }
    __device__ void finalize(const double* tot) const {
        sc->refresh = 0;
        fsai_beta(sc, tot[0]);
    }
};

struct EpiCgPqZ {
    static constexpr bool kPre = true;   // solver loops only
    static constexpr int NS = 1;
    float* q;
    const float* z;
    float* p0;                     // direction pair: p_k goes to p[k & 1]
    float* p1;
    const float* r0;               // residual pair and diagonal (Jacobi fallback)
    const float* r1;
    const float* dinv;
    DevScalars* sc;
    unsigned* counter;
    double* partials;
    const float* po = nullptr;     // per thread (begin)
    float* pn = nullptr;
    const float* rc = nullptr;
    float beta = 0.f;
    bool jac = false;
    __device__ bool active() const { return !sc->done && !sc->replace; }
    __device__ void tick() const {}
    __device__ void on_skip() const {}
    __device__ void begin() {
        const bool odd = sc->iter & 1;
        pn = odd ? p1 : p0;
        po = odd ? p0 : p1;
        rc = odd ? r1 : r0;
        beta = (float)sc->beta;
        jac = sc->mode == 1;
    }
    __device__ float gather(int c) const {
        const float zc = jac ? __ldg(rc + c) * __ldg(dinv + c) : __ldg(z + c);
        return beta != 0.f ? fmaf(beta, __ldg(po + c), zc) : zc;
    }
    __device__ void row(int i, float s, double* acc) const {
        const float zc = jac ? rc[i] * dinv[i] : z[i];
        const float pv = beta != 0.f ? fmaf(beta, po[i], zc) : zc;
        pn[i] = pv;
        q[i] = s;
        acc[0] += (double)pv * (double)s;
    }
    __device__ void finalize(const double* tot) const {
        const double pq = tot[0];
        sc->pq = pq;
        if (!(pq > 0.0) || !isfinite(pq)) {
            sc->breakdown = 1;
            sc->done = 1;
            sc->alpha = 0.0;
        } else {
            sc->alpha = sc->rz / pq;
        }
    }
};

template <bool IR>
struct EpiFsaiM {
    static constexpr bool kPre = true;   // solver loops only
    static constexpr int NS = 3;
    const float* r0;
    const float* r1;
    const float* q;
    const float* p0;
    const float* p1;
    std::conditional_t<IR, double, float>* x;
    const float* dinv;
    float* z;
    DevScalars* sc;
    unsigned* counter;
    double* partials;
    Ctx c;
    const float* rc = nullptr;     // per thread (begin)
    float* rn = nullptr;
    const float* pc = nullptr;
    double a = 0.0;
    float af = 0.f;
    __device__ bool active() const { return !sc->done && !sc->replace; }
    // last kernel of an iteration: watchdog (iterations that run), and the
    // loop condition in case this launch returns at once (the last CTA sets
    // it again below)
    __device__ void tick() const {
        const bool run = !sc->done && !sc->replace;
        if (run) loop_watchdog(sc);
        set_cond(c, run);
    }
    __device__ void on_skip() const {}
    __device__ void begin() {
        const bool odd = sc->iter & 1;
        rc = odd ? r1 : r0;
        rn = const_cast<float*>(odd ? r0 : r1);
        pc = odd ? p1 : p0;
        a = sc->alpha;
        af = (float)a;
    }
    __device__ float gather(int col) const { return fmaf(-af, __ldg(q + col), __ldg(rc + col)); }
    __device__ void row(int i, float s, double* acc) const {
        const float rv = fmaf(-af, q[i], rc[i]);
        rn[i] = rv;
        if constexpr (IR) x[i] = fma(a, (double)pc[i], x[i]);
        else x[i] = fmaf(af, pc[i], x[i]);
        z[i] = s;
        acc[0] += (double)rv * rv;
        if (dinv) acc[1] += (double)rv * rv * dinv[i];
        acc[2] += (double)rv * (double)s;
    }
    __device__ void finalize(const double* tot) const {
        DevScalars* s = sc;
        if constexpr (IR) {
            // a due replacement ends the loop of iterations; the step after
            // it (EpiReplace, EpiMzR) re-arms it
            cg_finalize_ir(s, tot[0], tot[1]);
            set_cond(c, !s->done && !s->replace);
            if (s->replace || s->done) return;
        } else {
            cg_finalize_xr(s, tot[0], tot[1]);
            set_cond(c, !s->done);
            if (s->done) return;
        }
        if (s->mode == 2) fsai_beta(s, tot[2]);
    }
};

// ============================ BiCGSTAB =====================================

static __device__ void bicg_init_scalars(const Ctx& c, const SolveParams* __restrict__ prm, int n,
                                         double bb);

static __global__ void __launch_bounds__(kNT)
bicg_init(const float4* __restrict__ b, float4* __restrict__ x, float4* __restrict__ r,
          float4* __restrict__ r0, float4* __restrict__ p, float4* __restrict__ v, int n4, int n,
          const SolveParams* __restrict__ prm, Ctx c) {
    pdl_begin();
    double acc[1] = {0.0};
    MPS_GRID_STRIDE(i, n4) {
        const float4 bv = b[i];
        x[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        v[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        r[i] = bv;
        r0[i] = bv;
        p[i] = bv;
        acc[0] += dot4(bv, bv);
    }
    double tot[1];
    if (!reduce_partials<1>(c, 4, acc, tot)) return;
    if (threadIdx.x != 0) return;
    bicg_init_scalars(c, prm, n, tot[0]);
}

// Scalars of a BiCGSTAB start from bb = ||b||^2 (one thread).
static __device__ void bicg_init_scalars(const Ctx& c, const SolveParams* __restrict__ prm, int n,
                                         double bb) {
    DevScalars* s = c.sc;
    s->n = n;
    s->compat = prm->compat;
    s->max_iter = prm->compat ? (n < 5000 ? n : 5000) : prm->max_iter;
    s->iter = 0;
    s->done = 0;
    s->converged = 0;
    s->breakdown = 0;
    s->stalled = 0;
    s->snapshot = 0;
    s->err = 0;
    s->bnorm2 = bb;
    s->tol2 = prm->tol * prm->tol * bb;
    // spmv.cpp:724,744-752: slots start at 1 and r.r is added on top (rho0 = 1 + b.b)
    s->rho = (prm->compat ? 1.0 : 0.0) + bb;
    s->rho_old = 1.0;
    s->alpha = 1.0;
    s->omega = 1.0;
    s->rnorm2 = bb;
    s->staged = 1e9;                                         // spmv.cpp:712
    s->beta = 0.0;
    s->guard = 0;
    s->guard_limit = s->max_iter + 8;
    s->rr_ref = bb;
    s->delta2 = prm->delta * prm->delta;
    s->replace = 0;
    s->replaced = 0;
    s->refresh = 0;
    if (!isfinite(bb)) {
        s->err = kErrNotFinite;
        s->done = 1;
    } else if (!prm->compat && bb == 0.0) {
        s->done = 1;
        s->converged = 1;
    } else if (s->max_iter <= 0) {
        s->done = 1;
    }
    set_cond(c, !s->done);
}

// upp (bicgstab.metal:12-68): p = r on the first iteration, else
// p = r + beta (p - omega v) with beta prepared by the previous iteration.
static __global__ void __launch_bounds__(kNT)
bicg_update_p(float4* __restrict__ p, const float4* __restrict__ r, const float4* __restrict__ v,
              int n4, Ctx c) {
    pdl_begin();
    DevScalars* s = c.sc;
    if (s->done) return;
    if (s->iter == 0) {
        MPS_GRID_STRIDE(i, n4) p[i] = r[i];
        return;
    }
    const float beta = (float)s->beta, omega = (float)s->omega;
    MPS_GRID_STRIDE(i, n4) {
        const float4 pv = p[i], vv = v[i], rv = r[i];
        const float4 t = axpy4(-omega, vv, pv);
        p[i] = axpy4(beta, t, rv);
    }
}

// v = A p ; sigma = r0.v ; alpha = rho / sigma (fused_spvmv + f_upalpha_ups)
struct EpiBicgV {
    static constexpr int NS = 1;
    float* v;
    const float* r0;
    DevScalars* sc;
    unsigned* counter;
    double* partials;
    __device__ bool active() const { return !sc->done; }
    __device__ void tick() const {}
    __device__ void on_skip() const {}
    __device__ void row(int r, float s, double* acc) const {
        v[r] = s;
        acc[0] += (double)r0[r] * (double)s;
    }
    __device__ void finalize(const double* tot) const {
        const double sigma = tot[0];
        sc->sigma = sigma;
        if (!sc->compat && (sigma == 0.0 || !isfinite(sigma))) {
            sc->breakdown = 1;
            sc->done = 1;
            sc->alpha = 0.0;
            return;
        }
        sc->alpha = sc->rho / sigma;                         // bicgstab.metal:87, unguarded
    }
};

// s = r - alpha v
static __global__ void __launch_bounds__(kNT)
bicg_update_s(float4* __restrict__ s_, const float4* __restrict__ r, const float4* __restrict__ v,
              int n4, Ctx c) {
    pdl_begin();
    if (c.sc->done) return;
    const float a = (float)c.sc->alpha;
    MPS_GRID_STRIDE(i, n4) s_[i] = axpy4(-a, v[i], r[i]);
}

// t = A s ; phi1 = t.s ; phi2 = t.t ; omega (spmv_op + f_dip)
struct EpiBicgT {
    static constexpr int NS = 2;
    float* t;
    const float* s_;
    DevScalars* sc;
    unsigned* counter;
    double* partials;
    __device__ bool active() const { return !sc->done; }
    __device__ void tick() const {}
    __device__ void on_skip() const {}
    __device__ void row(int r, float s, double* acc) const {
        t[r] = s;
        acc[0] += (double)s * (double)s_[r];
        acc[1] += (double)s * (double)s;
    }
    __device__ void finalize(const double* tot) const {
        sc->phi1 = tot[0];
        sc->phi2 = tot[1];
        sc->omega = fabs(tot[1]) < 1e-20 ? 0.0 : tot[0] / tot[1];   // bicgstab.metal:264-269
    }
};

// Stop rule and next beta of a BiCGSTAB iteration (outside reference_compat),
// once iter, rho_old, rho and rnorm2 hold the new values.
static __device__ void bicg_stop_beta(DevScalars* s) {
    if (!isfinite(s->rnorm2)) {
        s->breakdown = 1;
        s->done = 1;
    } else if (s->rnorm2 <= s->tol2) {
        s->converged = 1;
        s->done = 1;
    } else if (s->omega == 0.0 || s->rho == 0.0) {
        s->breakdown = 1;
        s->done = 1;
    } else if (s->iter >= s->max_iter) {
        s->done = 1;
    }
    s->beta = (s->rho / s->rho_old) * (s->alpha / s->omega);
}

// x += alpha p + omega s ; r = s - omega t ; rho = r0.r ; ||r||^2
// (f_upomega_upxr_laa, bicgstab.metal:245-326).  Last kernel of an iteration.
static __global__ void __launch_bounds__(kNT)
bicg_update_xr(float4* __restrict__ x, float4* __restrict__ r, const float4* __restrict__ p,
               const float4* __restrict__ r0, const float4* __restrict__ s_,
               const float4* __restrict__ t, float4* __restrict__ xsnap, int n4, Ctx c) {
    pdl_begin();
    DevScalars* s = c.sc;
    if (blockIdx.x == 0 && threadIdx.x == 0) loop_watchdog(s);
    if (s->done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_cond(c, false);
        return;
    }
    const int it = s->iter;   // 0-based index of this iteration
    // Reference-compat delayed stop (spmv.cpp:835-859): at a check index
    // other than 0, a staged ||r||^2 below 1e-5 returns the checkpoint.
    const bool check = s->compat && (it % 50 == 0);
    const bool stop_now = check && it > 0 && s->staged < 1e-5;
    const bool snap = check && !stop_now;
    const float a = (float)s->alpha, w = (float)s->omega;
    double acc[2] = {0.0, 0.0};
    if (!stop_now) {
        MPS_GRID_STRIDE(i, n4) {
            const float4 sv = s_[i], tv = t[i];
            float4 xv = axpy4(a, p[i], x[i]);
            xv = axpy4(w, sv, xv);
            x[i] = xv;
            if (snap) xsnap[i] = xv;
            const float4 rv = axpy4(-w, tv, sv);
            r[i] = rv;
            acc[0] += dot4(r0[i], rv);
            acc[1] += dot4(rv, rv);
        }
    }
    double tot[2];
    if (!reduce_partials<2>(c, 7, acc, tot)) return;
    if (threadIdx.x != 0) return;
    if (stop_now) {
        s->done = 1;
        s->converged = 1;
        s->snapshot = 1;
        s->rnorm2 = s->staged;
        s->iter = it - 50 + 1;
        set_cond(c, false);
        return;
    }
    s->iter = it + 1;
    s->rho_old = s->rho;
    s->rho = tot[0];
    s->rnorm2 = tot[1];
    if (s->compat) {
        double beta = 0.0;                                   // bicgstab.metal:46-56
        if (fabs(s->rho_old) > 1e-15 && fabs(s->omega) > 1e-15) {
            beta = (s->rho / s->rho_old) * (s->alpha / s->omega);
            if (isinf(beta) || isnan(beta)) beta = 0.0;
        }
        s->beta = beta;
        if (check) s->staged = tot[1];
        if (s->iter >= s->max_iter) s->done = 1;
    } else {
        bicg_stop_beta(s);
    }
    set_cond(c, !s->done);
}

// ============================ Richardson ===================================

// The solver scalars at the start (x = 0, ||b||^2 = bb); shared by the graph
// form (rich_init) and the persistent form.
__device__ __forceinline__ void rich_init_scalars(DevScalars* s, const SolveParams* prm, int n, double bb);

// One row of x_out = x_in + (w b + (-w) A x_in): iterative_step's spmv_op and
// two weighted_adds (richardson/spmv.cpp:376-495), each product and sum
// rounded to FP32 on its own (no contraction), in both forms.
__device__ __forceinline__ float rich_update(float xin, float w, float bv, float ax) {
    return __fadd_rn(xin, __fadd_rn(__fmul_rn(w, bv), __fmul_rn(-w, ax)));
}

// Iteration count and stop rule after ||b - A x_in||^2 = rr.
__device__ __forceinline__ void rich_finalize(DevScalars* sc, double rr) {
    const int it = ++sc->iter;
    sc->rnorm2 = rr;
    if (sc->tol2 > 0.0 && rr <= sc->tol2) {
        sc->converged = 1;
        sc->done = 1;
    }
    if (it >= sc->max_iter) sc->done = 1;
}

static __global__ void __launch_bounds__(kNT)
rich_init(const float4* __restrict__ b, float4* __restrict__ x0, int n4, int n,
          const SolveParams* __restrict__ prm, Ctx c) {
    pdl_begin();
    double acc[1] = {0.0};
    MPS_GRID_STRIDE(i, n4) {
        const float4 bv = b[i];
        x0[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        acc[0] += dot4(bv, bv);
    }
    double tot[1];
    if (!reduce_partials<1>(c, 8, acc, tot)) return;
    if (threadIdx.x != 0) return;
    rich_init_scalars(c.sc, prm, n, tot[0]);
    set_cond(c, !c.sc->done);
}

__device__ __forceinline__ void rich_init_scalars(DevScalars* s, const SolveParams* prm, int n, double bb) {
    s->n = n;
    s->compat = prm->compat;
    s->max_iter = prm->compat ? 1000 : prm->max_iter;        // richardson/spmv.cpp:402
    s->omega_rich = prm->compat ? 0.01 : prm->omega;
    s->iter = 0;
    s->done = 0;
    s->converged = 0;
    s->breakdown = 0;
    s->snapshot = 0;
    s->err = 0;
    s->bnorm2 = bb;
    s->rnorm2 = bb;
    s->tol2 = prm->compat ? 0.0 : prm->tol * prm->tol * bb;
    s->guard = 0;
    s->guard_limit = s->max_iter / 2 + 8;
    if (!isfinite(bb)) {
        s->err = kErrNotFinite;
        s->done = 1;
    } else if (s->max_iter <= 0) {
        s->done = 1;
    }
}

// x_out = x_in + (w b + (-w) A x_in)  (iterative_step's spmv_op + two
// weighted_add, fused); ||b - A x_in||^2 for the optional stop test.
struct EpiRich {
    static constexpr int NS = 1;
    const float* xin;
    float* xout;
    const float* b;
    DevScalars* sc;
    unsigned* counter;
    double* partials;
    Ctx ctx;
    int last_in_body;
    __device__ void tick() const {
        if (last_in_body) loop_watchdog(sc);
    }
    __device__ bool active() const { return !sc->done; }
    __device__ void on_skip() const {
        if (last_in_body) set_cond(ctx, false);
    }
    __device__ void row(int r, float s, double* acc) const {
        const float w = (float)__ldcg(&sc->omega_rich);
        const float bv = b[r];
        xout[r] = rich_update(xin[r], w, bv, s);
        const double res = (double)bv - (double)s;
        acc[0] += res * res;
    }
    __device__ void finalize(const double* tot) const {
        rich_finalize(sc, tot[0]);
        if (last_in_body) set_cond(ctx, !sc->done);
    }
};

// Result selection without a host round-trip.
enum { kResX = 0, kResRich = 1 };
static __global__ void copy_result(const float* __restrict__ x0, const float* __restrict__ x1,
                            const float* __restrict__ xsnap, float* __restrict__ out, int n,
                            int kind, const DevScalars* __restrict__ sc) {
    pdl_begin();
    const float* src = x0;
    if (kind == kResRich)
        src = (sc->iter & 1) ? x1 : x0;
    else if (sc->snapshot)
        src = xsnap;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = src[i];
}

}  // namespace mps
