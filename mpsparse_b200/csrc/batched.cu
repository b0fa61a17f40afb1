// batched.cu -- thousands of independent SPD systems in one persistent launch.
//
// The systems are stacked into one block-diagonal CSR (global row and column
// indices; system s owns rows [row_off[s], row_off[s+1])).  A persistent
// kernel of 512-thread CTAs splits each CTA into groups of WPS warps; every
// group takes the next system from a queue ordered largest-first (longest
// processing time first, so the big systems do not finish last) and runs PCG
// on it to convergence with group-level barriers only (named barriers, or
// __syncwarp when a group is one warp): no grid-wide synchronisation, no host
// round trip.  Per system: preconditioner none / Jacobi / learned FSAI (with
// the same stall watch and Jacobi fallback as the single-system solver), and a
// convergence record (iterations, converged flag, relative residual) -- the
// per-system convergence mask.  WPS (warps per system, hence rows per warp)
// is chosen by the autotuner, which times whole-batch launches.  Systems of
// at least kBigRows rows can instead be solved by a whole thread-block
// cluster each (8 CTAs, 4096 threads; cluster barriers and distributed
// shared memory for the reductions) in a second persistent kernel beside the
// warp groups; the autotuner keeps that path only when the batch is faster
// with it.  No reference counterpart (the reference solves one system per
// call).
#include <cooperative_groups.h>

#include <algorithm>
#include <chrono>
#include <numeric>
#include <type_traits>
#include <vector>

#include "handles.hpp"

namespace mps {
namespace {

constexpr int kBatchNT = 512;

struct BatchDev {
    const int* rp;
    const int* ci;
    const float* v;
    const int* grp;       // G (learned factor), may be null
    const int* gci;
    const float* gv;
    const int* gtrp;      // G^T
    const int* gtci;
    const float* gtv;
    const float* dinv;
    const int* row_off;   // n_sys + 1
    const int* order;     // queue order (largest first)
    const signed char* kind;   // per system: 0 none, 1 Jacobi, 2 FSAI, 3 skip
    int n_sys;            // systems in the queue
    float* r;
    float* p;
    float* q;
    float* w;
};

struct BatchOut {
    int* iters;
    int* converged;
    float* relres;
};

template <int WPS>
__device__ __forceinline__ void group_sync(int g) {
    if (WPS == 1) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(WPS * 32) : "memory");
    }
}

// Sum NS doubles over the group (fixed order: every thread gets the same bits).
template <int WPS, int NS>
__device__ __forceinline__ void group_reduce(double* v, double (*red)[4], int g, int lt) {
#pragma unroll
    for (int i = 0; i < NS; ++i) v[i] = warp_sum(v[i]);
    const int w = lt >> 5;
    if ((lt & 31) == 0)
#pragma unroll
        for (int i = 0; i < NS; ++i) red[w][i] = v[i];
    group_sync<WPS>(g);
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < WPS; ++k) s += red[k][i];
        v[i] = s;
    }
    group_sync<WPS>(g);
}

// A solving group: WPS warps of one 512-thread CTA (WarpGroup), or the
// whole of a CS-CTA thread-block cluster (ClusterGroup, for the largest
// systems).  Both provide the group size, the thread's rank in the group, a
// group barrier, a fixed-order FP64 all-reduce and the queue pop.
struct GroupShared {
    double red[32][4];                 // per-warp partial sums (up to 1024 threads)
    double cred[2][16][4];             // cluster: per-CTA partials (double-buffered)
    int next[32];
    int flip;
};

template <int WPS>
struct WarpGroup {
    static constexpr int GS = WPS * 32;
    int g, lt;
    __device__ WarpGroup() : g(threadIdx.x / GS), lt(threadIdx.x % GS) {}
    __device__ void sync() const { group_sync<WPS>(g); }
    template <int NS>
    __device__ void reduce(double* v, GroupShared& sh) const {
        group_reduce<WPS, NS>(v, reinterpret_cast<double(*)[4]>(&sh.red[g * WPS][0]), g, lt);
    }
    __device__ int pop(unsigned* queue, GroupShared& sh) const {
        if (lt == 0) sh.next[g] = (int)atomicAdd(queue, 1u);
        sync();
        const int q = sh.next[g];
        sync();
        return q;
    }
    __device__ float gather(const float* x, int c) const { return x[c]; }
    __device__ double gather64(const double* x, int c) const { return x[c]; }
};

template <int CS>
struct ClusterGroup {
    static constexpr int GS = CS * kBatchNT;
    int lt;
    unsigned rank;
    __device__ ClusterGroup() {
        rank = cooperative_groups::this_cluster().block_rank();
        lt = (int)rank * kBatchNT + threadIdx.x;
    }
    __device__ void sync() const { cooperative_groups::this_cluster().sync(); }
    template <int NS>
    __device__ void reduce(double* v, GroupShared& sh) const {
        auto cl = cooperative_groups::this_cluster();
        // CTA sums in a fixed order
#pragma unroll
        for (int i = 0; i < NS; ++i) v[i] = warp_sum(v[i]);
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0)
#pragma unroll
            for (int i = 0; i < NS; ++i) sh.red[w][i] = v[i];
        __syncthreads();
        const int buf = sh.flip;
        if (threadIdx.x == 0) {
            double* dst = cl.map_shared_rank(&sh.cred[buf][rank][0], 0);
#pragma unroll
            for (int i = 0; i < NS; ++i) {
                double s = 0.0;
                for (int k = 0; k < kBatchNT / 32; ++k) s += sh.red[k][i];
                dst[i] = s;
            }
        }
        cl.sync();   // partials of every CTA are in CTA 0's shared memory
        const double* src = cl.map_shared_rank(&sh.cred[buf][0][0], 0);
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < CS; ++k) s += src[k * 4 + i];
            v[i] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) sh.flip = buf ^ 1;
        __syncthreads();
    }
    __device__ int pop(unsigned* queue, GroupShared& sh) const {
        auto cl = cooperative_groups::this_cluster();
        if (rank == 0 && threadIdx.x == 0) sh.next[0] = (int)atomicAdd(queue, 1u);
        cl.sync();
        const int q = *cl.map_shared_rank(&sh.next[0], 0);
        cl.sync();   // rank 0 may overwrite next[0] only after every CTA read it
        return q;
    }
    // vectors written by other CTAs of the cluster: read through L2
    __device__ float gather(const float* x, int c) const { return __ldcg(x + c); }
    __device__ double gather64(const double* x, int c) const { return __ldcg(x + c); }
};

// Rows i and j of a CSR times x through the group's gather (see row_dot2).
template <class Grp>
__device__ __forceinline__ void grp_dot2(const Grp& G, const int* __restrict__ rp,
                                         const int* __restrict__ ci, const float* __restrict__ v,
                                         const float* x, int i, int j, bool has_j, float& s0,
                                         float& s1) {
    const int b0 = __ldg(rp + i), e0 = __ldg(rp + i + 1);
    const int b1 = has_j ? __ldg(rp + j) : 0, e1 = has_j ? __ldg(rp + j + 1) : 0;
    s0 = 0.f;
    s1 = 0.f;
    const int len = max(e0 - b0, e1 - b1);
    for (int k = 0; k < len; k += 4) {
        float x0[4], x1[4], v0[4], v1[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const bool in0 = b0 + k + u < e0, in1 = b1 + k + u < e1;
            const int c0 = in0 ? __ldg(ci + b0 + k + u) : 0;
            const int c1 = in1 ? __ldg(ci + b1 + k + u) : 0;
            v0[u] = in0 ? __ldg(v + b0 + k + u) : 0.f;
            v1[u] = in1 ? __ldg(v + b1 + k + u) : 0.f;
            x0[u] = in0 ? G.gather(x, c0) : 0.f;
            x1[u] = in1 ? G.gather(x, c1) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (b0 + k + u < e0) s0 = fmaf(v0[u], x0[u], s0);
            if (b1 + k + u < e1) s1 = fmaf(v1[u], x1[u], s1);
        }
    }
}

// Rows lo + lt, lo + lt + GS, ... of a CSR times x, two rows (i, i + GS)
// per trip as grp_dot2 does, with the next pair's row bounds loaded before
// this pair's products (one dependent memory round trip less per trip);
// emit(row, sum) in row order.
template <class Grp, class F>
__device__ __forceinline__ void grp_spmv_rows(const Grp& G, const int* __restrict__ rp,
                                              const int* __restrict__ ci, const float* __restrict__ v,
                                              const float* x, int lo, int hi, F emit) {
    constexpr int GS = Grp::GS;
    int i = lo + G.lt;
    if (i >= hi) return;
    int j = i + GS;
    int b0 = __ldg(rp + i), e0 = __ldg(rp + i + 1);
    int b1 = j < hi ? __ldg(rp + j) : 0, e1 = j < hi ? __ldg(rp + j + 1) : 0;
    for (;;) {
        const int in = i + 2 * GS, jn = in + GS;
        const int nb0 = in < hi ? __ldg(rp + in) : 0, ne0 = in < hi ? __ldg(rp + in + 1) : 0;
        const int nb1 = jn < hi ? __ldg(rp + jn) : 0, ne1 = jn < hi ? __ldg(rp + jn + 1) : 0;
        float s0 = 0.f, s1 = 0.f;
        const int len = max(e0 - b0, e1 - b1);
        for (int k = 0; k < len; k += 4) {
            float x0[4], x1[4], v0[4], v1[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const bool in0 = b0 + k + u < e0, in1 = b1 + k + u < e1;
                const int c0 = in0 ? __ldg(ci + b0 + k + u) : 0;
                const int c1 = in1 ? __ldg(ci + b1 + k + u) : 0;
                v0[u] = in0 ? __ldg(v + b0 + k + u) : 0.f;
                v1[u] = in1 ? __ldg(v + b1 + k + u) : 0.f;
                x0[u] = in0 ? G.gather(x, c0) : 0.f;
                x1[u] = in1 ? G.gather(x, c1) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (b0 + k + u < e0) s0 = fmaf(v0[u], x0[u], s0);
                if (b1 + k + u < e1) s1 = fmaf(v1[u], x1[u], s1);
            }
        }
        emit(i, s0);
        if (j < hi) emit(j, s1);
        if (in >= hi) break;
        i = in;
        j = jn;
        b0 = nb0;
        e0 = ne0;
        b1 = nb1;
        e1 = ne1;
    }
}

// b_i - (A x)_i in FP64 for an FP64 x (exact products of the FP32 values).
template <class Grp>
__device__ __forceinline__ double grp_resid64(const Grp& G, const int* __restrict__ rp,
                                              const int* __restrict__ ci, const float* __restrict__ v,
                                              const double* x, float bi, int i) {
    const int e = __ldg(rp + i + 1);
    double s = 0.0;
    for (int k = __ldg(rp + i); k < e; ++k) s = fma((double)__ldg(v + k), G.gather64(x, __ldg(ci + k)), s);
    return (double)bi - s;
}

// PCG on the systems the queue hands out, one system per group at a time.
// XT = float: x in FP32, a system stops when its recurrence residual meets
// tol.  XT = double (mixed precision): x accumulated in FP64, and whenever a
// system's recurrence residual has dropped by sqrt(delta2) since the last
// replacement, or meets tol, it is replaced by the FP64 b - A x (reliable
// updates, as in the single-system solver); the system stops only when that
// true residual meets tol, and relres reports it.
template <class Grp, typename XT>
__device__ __forceinline__ void batch_pcg_body(const BatchDev& B, const float* __restrict__ b,
                                               XT* __restrict__ x, const BatchOut& out, double tol,
                                               int max_iter, int stall_window, unsigned* queue,
                                               GroupShared& sh, double delta2) {
    constexpr bool kIR = std::is_same<XT, double>::value;
    const Grp G;
    constexpr int GS = Grp::GS;
    const int lt = G.lt;
    for (;;) {
        const int qi = G.pop(queue, sh);
        if (qi >= B.n_sys) break;
        const int sys = B.order[qi];
        const int lo = B.row_off[sys], hi = B.row_off[sys + 1];
        int mode = B.kind[sys];
        if (mode == 3) {                          // masked out: x untouched
            if (lt == 0) {
                out.iters[sys] = 0;
                out.converged[sys] = 0;
                out.relres[sys] = -1.f;
            }
            continue;
        }
        // init: x = 0, r = b, p = M b
        double acc[2] = {0.0, 0.0};
        for (int i = lo + lt; i < hi; i += GS) {
            const float bi = b[i];
            x[i] = XT(0);
            B.r[i] = bi;
            const float z = mode == 1 ? bi * B.dinv[i] : bi;
            if (mode != 2) B.p[i] = z;
            acc[0] += (double)bi * bi;
            acc[1] += (double)bi * z;
        }
        G.template reduce<2>(acc, sh);
        const double bb = acc[0];
        double rz = acc[1], rr = bb;
        const double thresh = tol * tol * bb;
        int it = 0, conv = bb == 0.0, best_it = 0;
        double best = 1e300, rr_ref = bb;
        if (!conv && mode == 2) {                 // p = G^T G b
            double a2[1] = {0.0};
            for (int i = lo + lt; i < hi; i += 2 * GS) {
                const int j = i + GS;
                float w0, w1;
                grp_dot2(G, B.grp, B.gci, B.gv, B.r, i, j, j < hi, w0, w1);
                B.w[i] = w0;
                a2[0] += (double)w0 * w0;
                if (j < hi) {
                    B.w[j] = w1;
                    a2[0] += (double)w1 * w1;
                }
            }
            G.template reduce<1>(a2, sh);
            rz = a2[0];
            for (int i = lo + lt; i < hi; i += 2 * GS) {
                const int j = i + GS;
                float z0, z1;
                grp_dot2(G, B.gtrp, B.gtci, B.gtv, B.w, i, j, j < hi, z0, z1);
                B.p[i] = z0;
                if (j < hi) B.p[j] = z1;
            }
            G.sync();
        }
        while (!conv && it < max_iter) {
            double a[1] = {0.0};
            grp_spmv_rows(G, B.rp, B.ci, B.v, B.p, lo, hi, [&](int i, float qi) {
                B.q[i] = qi;
                a[0] += (double)B.p[i] * qi;
            });
            G.template reduce<1>(a, sh);
            if (!(a[0] > 0.0)) break;             // breakdown (not SPD)
            const double alpha64 = rz / a[0];
            const float alpha = (float)alpha64;
            double c[2] = {0.0, 0.0};
            // four rows per thread per trip, every load issued before the
            // first store (one memory round trip per trip, not per row);
            // rows are visited, and summed, in the same order as one at a time
            constexpr int UV = 4;
            for (int i0 = lo + lt; i0 < hi; i0 += UV * GS) {
                float pv[UV], qv[UV], rv[UV], dv[UV];
                XT xv[UV];
#pragma unroll
                for (int u = 0; u < UV; ++u) {
                    const int i = i0 + u * GS;
                    if (i < hi) {
                        pv[u] = B.p[i];
                        qv[u] = B.q[i];
                        rv[u] = B.r[i];
                        dv[u] = B.dinv[i];
                        xv[u] = x[i];
                    }
                }
#pragma unroll
                for (int u = 0; u < UV; ++u) {
                    const int i = i0 + u * GS;
                    if (i < hi) {
                        if constexpr (kIR) x[i] = fma(alpha64, (double)pv[u], xv[u]);
                        else x[i] = fmaf(alpha, pv[u], xv[u]);
                        const float ri = fmaf(-alpha, qv[u], rv[u]);
                        B.r[i] = ri;
                        c[0] += (double)ri * ri;
                        c[1] += (double)ri * ri * dv[u];
                    }
                }
            }
            G.template reduce<2>(c, sh);
            ++it;
            rr = c[0];
            if constexpr (kIR) {
                if (rr <= thresh || rr < delta2 * rr_ref) {
                    // residual replacement: r = (float)(b - A x) from the FP64 x
                    double t[2] = {0.0, 0.0};
                    for (int i = lo + lt; i < hi; i += GS) {
                        const double rt = grp_resid64(G, B.rp, B.ci, B.v, x, b[i], i);
                        const float rf = (float)rt;
                        B.r[i] = rf;
                        t[0] += rt * rt;
                        t[1] += (double)rf * rf * B.dinv[i];
                    }
                    G.template reduce<2>(t, sh);
                    c[0] = t[0];
                    c[1] = t[1];
                    rr = t[0];
                    rr_ref = t[0];
                }
            }
            if (rr <= thresh) {
                conv = 1;
                break;
            }
            double beta;
            if (mode == 2) {
                double d[1] = {0.0};
                grp_spmv_rows(G, B.grp, B.gci, B.gv, B.r, lo, hi, [&](int i, float wi) {
                    B.w[i] = wi;
                    d[0] += (double)wi * wi;
                });
                G.template reduce<1>(d, sh);
                if (stall_window > 0 && !(d[0] < 0.25 * best) && it - best_it >= stall_window) {
                    mode = 1;                     // stalled: Jacobi from here, restart p
                    rz = c[1];
                    for (int i = lo + lt; i < hi; i += GS) B.p[i] = B.r[i] * B.dinv[i];
                    G.sync();
                    continue;
                }
                if (d[0] < 0.25 * best) {
                    best = d[0];
                    best_it = it;
                }
                beta = d[0] / rz;
                rz = d[0];
                const float bf = (float)beta;
                grp_spmv_rows(G, B.gtrp, B.gtci, B.gtv, B.w, lo, hi,
                              [&](int i, float zi) { B.p[i] = fmaf(bf, B.p[i], zi); });
            } else {
                const double rzn = mode == 1 ? c[1] : c[0];
                beta = rzn / rz;
                rz = rzn;
                const float bf = (float)beta;
                constexpr int UP = 4;
                for (int i0 = lo + lt; i0 < hi; i0 += UP * GS) {
                    float pv[UP], zv[UP];
#pragma unroll
                    for (int u = 0; u < UP; ++u) {
                        const int i = i0 + u * GS;
                        if (i < hi) {
                            pv[u] = B.p[i];
                            zv[u] = mode == 1 ? B.r[i] * B.dinv[i] : B.r[i];
                        }
                    }
#pragma unroll
                    for (int u = 0; u < UP; ++u) {
                        const int i = i0 + u * GS;
                        if (i < hi) B.p[i] = fmaf(bf, pv[u], zv[u]);
                    }
                }
            }
            G.sync();
        }
        if (lt == 0) {
            out.iters[sys] = it;
            out.converged[sys] = conv;
            out.relres[sys] = bb > 0.0 ? (float)sqrt(rr / bb) : 0.f;
        }
        G.sync();   // the next pop must not race this system's last reads
    }
}

template <int WPS, typename XT>
__global__ void __launch_bounds__(kBatchNT, 2)
batch_pcg(BatchDev B, const float* __restrict__ b, XT* __restrict__ x, BatchOut out, double tol,
          int max_iter, int stall_window, unsigned* queue, double delta2) {
    __shared__ GroupShared sh;
    batch_pcg_body<WarpGroup<WPS>, XT>(B, b, x, out, tol, max_iter, stall_window, queue, sh, delta2);
}

// 32 warps per system: one 1024-thread CTA per system.
template <typename XT>
__global__ void __launch_bounds__(1024, 1)
batch_pcg_cta(BatchDev B, const float* __restrict__ b, XT* __restrict__ x, BatchOut out,
              double tol, int max_iter, int stall_window, unsigned* queue, double delta2) {
    __shared__ GroupShared sh;
    batch_pcg_body<WarpGroup<32>, XT>(B, b, x, out, tol, max_iter, stall_window, queue, sh, delta2);
}

// One cluster of kClusterCTAs CTAs per system (launched with the cluster
// dimension attribute); every CTA of a cluster runs the same control flow,
// so every cluster barrier is reached by all of them.
constexpr int kClusterCTAs = 8;

template <typename XT>
__global__ void __launch_bounds__(kBatchNT, 2)
batch_pcg_cluster(BatchDev B, const float* __restrict__ b, XT* __restrict__ x, BatchOut out,
                  double tol, int max_iter, int stall_window, unsigned* queue, double delta2) {
    __shared__ GroupShared sh;
    if (threadIdx.x == 0) sh.flip = 0;
    cooperative_groups::this_cluster().sync();
    batch_pcg_body<ClusterGroup<kClusterCTAs>, XT>(B, b, x, out, tol, max_iter, stall_window, queue, sh,
                                                   delta2);
    cooperative_groups::this_cluster().sync();   // no CTA leaves while another reads its memory
}

template <typename XT>
using BatchKernel = void (*)(BatchDev, const float*, XT*, BatchOut, double, int, int, unsigned*, double);

template <typename XT>
BatchKernel<XT> batch_kernel(int wps) {
    switch (wps) {
        case 1: return batch_pcg<1, XT>;
        case 2: return batch_pcg<2, XT>;
        case 4: return batch_pcg<4, XT>;
        case 8: return batch_pcg<8, XT>;
        case 16: return batch_pcg<16, XT>;
        default: return batch_pcg_cta<XT>;
    }
}

int batch_threads(int wps) { return wps >= 32 ? 1024 : kBatchNT; }

}  // namespace
}  // namespace mps

using namespace mps;

struct mps_batch {
    mps_csr* A = nullptr;          // the block-diagonal matrix (owns G/G^T/diagonal)
    int n_sys = 0;
    std::vector<int> row_off;      // host copy
    int* d_row_off = nullptr;
    int* d_order = nullptr;
    signed char* d_kind = nullptr;
    float* d_work = nullptr;       // r, p, q, w
    unsigned* d_queue = nullptr;   // [0] warp groups, [1] clusters
    int wps = 16;
    // systems with at least kBigRows rows go to one thread-block cluster each
    int n_big = 0;
    int clusters = 0;              // the cluster kernel takes this many of the largest systems
    cudaStream_t side = nullptr;   // the cluster kernel's branch
    cudaEvent_t fork = nullptr, join = nullptr;
    // one-launch graph of the last call: [queue reset, persistent kernel]
    cudaGraphExec_t exec = nullptr;
    const void* exec_key[5] = {};
    int exec_mode = 0;             // 0: FP32 x, 1: mixed precision (FP64 x)
    double exec_delta2 = -1.0;
    int exec_wps = 0;
    int exec_clusters = -1;
    double exec_tol = -1.0;
    int exec_max_iter = -1;
    cudaStream_t cap = nullptr;
};

// Rows from which a system is solved by a cluster of kClusterCTAs CTAs
// (4096 threads, at least 4 rows each) rather than by warps of one CTA.
constexpr int kBigRows = 16384;

static BatchDev batch_view(mps_batch* B) {
    mps_csr* h = B->A;
    const size_t n = h->A.n_rows;
    BatchDev d{};
    d.rp = h->A.rp;
    d.ci = h->A.ci;
    d.v = h->A.v;
    if (h->has_fsai) {
        d.grp = h->G.rp;
        d.gci = h->G.ci;
        d.gv = h->G.v;
        d.gtrp = h->Gt.rp;
        d.gtci = h->Gt.ci;
        d.gtv = h->Gt.v;
    }
    d.dinv = h->H.dinv;
    d.row_off = B->d_row_off;
    d.order = B->d_order;
    d.kind = B->d_kind;
    d.n_sys = B->n_sys;
    d.r = B->d_work;
    d.p = B->d_work + (n + 4);
    d.q = B->d_work + 2 * (n + 4);
    d.w = B->d_work + 3 * (n + 4);
    return d;
}

// One batch: the largest systems (queue order front) on clusters in a side
// branch, the rest on warp groups, both persistent and fed by their queues.
template <typename XT>
static mps_status batch_launch(mps_batch* B, int wps, const float* b, XT* x,
                               double tol, int max_iter, int stall_window, BatchOut out,
                               cudaStream_t s, int use_clusters, double delta2 = 0.0) {
    BatchDev all = batch_view(B);
    const int nb = std::min(std::max(use_clusters, 0), B->n_big);
    MPS_CUDA(cudaMemsetAsync(B->d_queue, 0, 2 * sizeof(unsigned), s));
    if (nb > 0) {
        BatchDev big = all;
        big.n_sys = nb;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = kClusterCTAs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.blockDim = dim3(kBatchNT);
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cfg.gridDim = dim3(kClusterCTAs);
        int max_clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&max_clusters, batch_pcg_cluster<XT>, &cfg) != cudaSuccess ||
            max_clusters < 1)
            return cuda_fail(cudaGetLastError(), "cluster occupancy");
        // half of the GPU's clusters at most: the warp groups run beside them
        int nc = std::min(nb, std::max(1, max_clusters / 2));
        cfg.gridDim = dim3(nc * kClusterCTAs);
        cfg.stream = B->side;
        MPS_CUDA(cudaEventRecord(B->fork, s));
        MPS_CUDA(cudaStreamWaitEvent(B->side, B->fork, 0));
        MPS_CUDA(cudaLaunchKernelEx(&cfg, batch_pcg_cluster<XT>, big, b, x, out, tol, max_iter, stall_window,
                                    B->d_queue + 1, delta2));
        MPS_CUDA(cudaEventRecord(B->join, B->side));
    }
    BatchDev small = all;
    small.order = all.order + nb;
    small.n_sys = all.n_sys - nb;
    if (small.n_sys > 0) {
        BatchKernel<XT> k = batch_kernel<XT>(wps);
        const int nt = batch_threads(wps);
        int per_sm = resident_ctas(reinterpret_cast<const void*>(k), nt, 0);
        const int grid = num_sms() * (per_sm > 0 ? per_sm : 1);
        k<<<grid, nt, 0, s>>>(small, b, x, out, tol, max_iter, stall_window, B->d_queue, delta2);
        MPS_CUDA(cudaGetLastError());
    }
    if (nb > 0) MPS_CUDA(cudaStreamWaitEvent(s, B->join, 0));
    return MPS_OK;
}

extern "C" {

mps_status mps_batch_create(const int32_t* d_row_ptr, const int32_t* d_col_ind, const float* d_vals,
                            uint64_t nnz, uint32_t total_rows, const int32_t* h_row_off,
                            int32_t n_systems, mps_batch** out, cudaStream_t s) {
    if (!out || !h_row_off || n_systems <= 0) return fail(MPS_ERR_ARG, "bad batch arguments");
    *out = nullptr;
    if (h_row_off[0] != 0 || (uint32_t)h_row_off[n_systems] != total_rows)
        return fail(MPS_ERR_ARG, "row_off must start at 0 and end at total_rows");
    for (int i = 0; i < n_systems; ++i)
        if (h_row_off[i + 1] < h_row_off[i]) return fail(MPS_ERR_ARG, "row_off must be ascending");
    mps_batch* B = new mps_batch();
    mps_status st = mps_csr_create_from_csr(d_row_ptr, d_col_ind, d_vals, total_rows, total_rows, nnz,
                                            &B->A, s);
    if (st != MPS_OK) {
        delete B;
        return st;
    }
    B->n_sys = n_systems;
    B->row_off.assign(h_row_off, h_row_off + n_systems + 1);
    // largest first
    std::vector<int> order(n_systems);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (h_row_off[a + 1] - h_row_off[a]) > (h_row_off[b + 1] - h_row_off[b]);
    });
    auto rows_of = [&](int sy) { return h_row_off[sy + 1] - h_row_off[sy]; };
    while (B->n_big < n_systems && rows_of(order[B->n_big]) >= kBigRows) ++B->n_big;
    cudaError_t e = cudaSuccess;
    const size_t n = total_rows;
    if (e == cudaSuccess) e = cudaMalloc(&B->d_row_off, (n_systems + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&B->d_order, n_systems * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&B->d_kind, n_systems);
    if (e == cudaSuccess) e = cudaMalloc(&B->d_work, 4 * (n + 4) * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&B->d_queue, 2 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&B->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->join, cudaEventDisableTiming);
    if (e == cudaSuccess)
        e = cudaMemcpy(B->d_row_off, h_row_off, (n_systems + 1) * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(B->d_order, order.data(), n_systems * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(B->d_kind, 1, n_systems);   // Jacobi by default
    if (e != cudaSuccess) {
        mps_batch_destroy(B);
        return cuda_fail(e, "batch_create");
    }
    // Jacobi diagonal of the whole batch
    mps_solve_opts o;
    mps_solve_opts_default(&o);
    o.precond = MPS_PRECOND_JACOBI;
    st = prepare_precond(B->A, &o, s);
    if (st != MPS_OK) {
        mps_batch_destroy(B);
        return st;
    }
    *out = B;
    return MPS_OK;
}

mps_status mps_batch_destroy(mps_batch* B) {
    if (!B) return MPS_OK;
    if (B->A) mps_csr_destroy(B->A);
    cudaFree(B->d_row_off);
    cudaFree(B->d_order);
    cudaFree(B->d_kind);
    cudaFree(B->d_work);
    cudaFree(B->d_queue);
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->cap) cudaStreamDestroy(B->cap);
    if (B->side) cudaStreamDestroy(B->side);
    if (B->fork) cudaEventDestroy(B->fork);
    if (B->join) cudaEventDestroy(B->join);
    delete B;
    return MPS_OK;
}

mps_status mps_batch_attach_fsai(mps_batch* B, const mps_fsai_model* m, cudaStream_t s) {
    if (!B || !m) return fail(MPS_ERR_ARG, "null argument");
    if (B->exec) {                     // the captured launch holds the old factor's pointers
        cudaGraphExecDestroy(B->exec);
        B->exec = nullptr;
    }
    const mps_status st = mps_fsai_attach(B->A, m, s);
    if (st != MPS_OK) return st;
    return mps_fsai_model_status(m, s);   // the batch solve does not read the handle's error words
}

mps_status mps_batch_set_precond(mps_batch* B, const int8_t* h_kind) {
    if (!B || !h_kind) return fail(MPS_ERR_ARG, "null argument");
    for (int i = 0; i < B->n_sys; ++i) {
        if (h_kind[i] < 0 || h_kind[i] > 3) return fail(MPS_ERR_ARG, "kind must be 0, 1, 2 or 3");
        if (h_kind[i] == 2 && !B->A->has_fsai) return fail(MPS_ERR_ARG, "FSAI requested without a factor");
    }
    MPS_CUDA(cudaMemcpy(B->d_kind, h_kind, B->n_sys, cudaMemcpyHostToDevice));
    return MPS_OK;
}

int32_t mps_batch_warps_per_system(const mps_batch* B) { return B ? B->wps : 0; }

mps_status mps_batch_autotune(mps_batch* B, const float* d_b, double tol, int32_t max_iter,
                              int32_t* h_chosen_wps, float* h_ms /* 6 candidates */, cudaStream_t s) {
    if (!B || !d_b) return fail(MPS_ERR_ARG, "null argument");
    const size_t n = B->A->A.n_rows;
    float* xs = nullptr;
    int* it = nullptr;
    MPS_CUDA(cudaMalloc(&xs, n * sizeof(float)));
    MPS_CUDA(cudaMalloc(&it, 3 * B->n_sys * sizeof(int)));
    BatchOut o{it, it + B->n_sys, reinterpret_cast<float*>(it + 2 * B->n_sys)};
    const int cands[6] = {1, 2, 4, 8, 16, 32};
    if (h_ms)
        for (int c = 0; c < 6; ++c) h_ms[c] = 0.f;
    float best = 1e30f;
    int best_w = B->wps;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    mps_status st = MPS_OK;
    auto time_one = [&](int w, int cl) {
        float ms = 0.f;
        for (int rep = 0; rep < 1 && st == MPS_OK; ++rep) {
            cudaEventRecord(e0, s);
            st = batch_launch(B, w, d_b, xs, tol, max_iter, 400, o, s, cl);
            if (st != MPS_OK) break;
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms, e0, e1);
        }
        return ms;
    };
    // Timed on the whole batch (the balance between the largest systems'
    // latency and the bulk's throughput does not survive sampling): warps
    // per system from 16 down while the time improves, then the cluster
    // path for the largest systems on or off.
    (void)time_one(32, 0);                    // warm-up
    int cl = 0;
    float prev = 1e30f;
    for (int c = 5; c >= 0 && st == MPS_OK; --c) {
        const float ms = time_one(cands[c], 0);
        if (h_ms) h_ms[c] = ms;
        if (ms < best) {
            best = ms;
            best_w = cands[c];
        }
        if (ms > prev) break;                 // past the minimum
        prev = ms;
    }
    if (st == MPS_OK && B->n_big > 0) {
        // the largest systems on clusters: as many as one wave of clusters,
        // two, four, or all systems above kBigRows
        int max_clusters = 0;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = kClusterCTAs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.blockDim = dim3(kBatchNT);
        cfg.gridDim = dim3(kClusterCTAs);
        cfg.attrs = at;
        cfg.numAttrs = 1;
        if (cudaOccupancyMaxActiveClusters(&max_clusters, batch_pcg_cluster<float>, &cfg) != cudaSuccess) {
            cudaGetLastError();
            max_clusters = 0;
        }
        const int q = std::max(1, max_clusters / 2);
        const int ks[4] = {q, 2 * q, 4 * q, B->n_big};
        int last = 0;
        for (int i = 0; i < 4 && st == MPS_OK && max_clusters > 0; ++i) {
            const int k = std::min(ks[i], B->n_big);
            if (k <= last) continue;
            last = k;
            const float ms = time_one(best_w, k);
            if (ms < best) {
                best = ms;
                cl = k;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(xs);
    cudaFree(it);
    if (st != MPS_OK) return st;
    B->wps = best_w;
    B->clusters = cl;
    if (h_chosen_wps) *h_chosen_wps = best_w;
    return MPS_OK;
}

int32_t mps_batch_uses_clusters(const mps_batch* B) {
    return B ? std::min(std::max(B->clusters, 0), B->n_big) : 0;
}

mps_status mps_batch_set_clusters(mps_batch* B, int32_t n_systems) {
    if (!B) return fail(MPS_ERR_ARG, "null argument");
    B->clusters = n_systems < 0 ? B->n_big : n_systems;
    return MPS_OK;
}

}  // extern "C"

// The whole batch is one CUDA-graph launch (queue reset + persistent
// kernel), captured once per set of buffers and settings and reused.
template <typename XT>
static mps_status batch_solve(mps_batch* B, const float* d_b, XT* d_x, double tol, int32_t max_iter,
                              double delta2, int32_t* d_iters, int32_t* d_converged, float* d_relres,
                              cudaStream_t s) {
    if (!B || !d_b || !d_x || !d_iters || !d_converged || !d_relres)
        return fail(MPS_ERR_ARG, "null argument");
    BatchOut o{d_iters, d_converged, d_relres};
    tol = tol > 0 ? tol : 1e-6;
    max_iter = max_iter > 0 ? max_iter : 20000;
    const int mode = std::is_same<XT, double>::value ? 1 : 0;
    const void* key[5] = {d_b, d_x, d_iters, d_converged, d_relres};
    bool same = B->exec && B->exec_wps == B->wps && B->exec_clusters == B->clusters;
    for (int i = 0; i < 5 && same; ++i) same = key[i] == B->exec_key[i];
    same = same && B->exec_tol == tol && B->exec_max_iter == max_iter && B->exec_mode == mode &&
           B->exec_delta2 == delta2;
    if (!same) {
        if (B->exec) cudaGraphExecDestroy(B->exec);
        B->exec = nullptr;
        if (!B->cap) MPS_CUDA(cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking));
        MPS_CUDA(cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal));
        mps_status st = batch_launch(B, B->wps, d_b, d_x, tol, max_iter, 400, o, B->cap, B->clusters, delta2);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(B->cap, &g);
        if (st != MPS_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return cuda_fail(e, "batch graph capture");
        e = cudaGraphInstantiate(&B->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "batch graph instantiate");
        for (int i = 0; i < 5; ++i) B->exec_key[i] = key[i];
        B->exec_wps = B->wps;
        B->exec_clusters = B->clusters;
        B->exec_tol = tol;
        B->exec_max_iter = max_iter;
        B->exec_mode = mode;
        B->exec_delta2 = delta2;
    }
    MPS_CUDA(cudaGraphLaunch(B->exec, s));
    return MPS_OK;
}

extern "C" {

mps_status mps_batch_cg(mps_batch* B, const float* d_b, float* d_x, double tol, int32_t max_iter,
                        int32_t* d_iters, int32_t* d_converged, float* d_relres, cudaStream_t s) {
    return batch_solve<float>(B, d_b, d_x, tol, max_iter, 0.0, d_iters, d_converged, d_relres, s);
}

mps_status mps_batch_cg_mixed(mps_batch* B, const float* d_b, double* d_x64, double tol, double inner_tol,
                              int32_t max_iter, int32_t* d_iters, int32_t* d_converged, float* d_relres,
                              cudaStream_t s) {
    if (!(inner_tol > 0.0) || !(inner_tol < 1.0)) inner_tol = 1e-3;
    return batch_solve<double>(B, d_b, d_x64, tol, max_iter, inner_tol * inner_tol, d_iters, d_converged,
                               d_relres, s);
}

}  // extern "C"
