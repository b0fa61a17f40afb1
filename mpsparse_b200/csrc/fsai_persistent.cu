// fsai_persistent.cu -- whole solves as one cooperative kernel, for matrices
// whose share of one CTA per SM (its rows, their vector window, or both)
// fits that CTA's shared memory: reliable-update
// FSAI-PCG (product form: z = M r with M = G^T G; fsai_pcg_persistent),
// plain CG / Jacobi-PCG, FP32 or with reliable updates (cg_persistent), and
// BiCGSTAB (bicg_persistent).
//
// The graph form of the same solve (driver.hpp, build_graph_nested) runs two
// grid-wide kernels per iteration; on an L2-resident system (512^2: 1.3 M
// nonzeros in A, 1.8 M in M) each kernel is bound by its fixed latency --
// launch, tile copies, the last-CTA reduction -- not by bytes.  Here one CTA
// per SM owns a block of rows of A and of M for the whole solve (held in its
// shared memory, except in the stream form) and the two dependent steps of
// an iteration are separated by grid barriers instead of kernel boundaries:
//   step 1  p = z + beta p_old, q = A p, p.q                          -> alpha
//   step 2  x += alpha p (FP64), r' = r - alpha q, z = M r',
//           r'.r', r'.D^-1 r', r'.z                                  -> beta
// plus, when due, the residual replacement r = (float)(b - A x) in FP64 and
// z = M r.  In the window form each step first stages its multiplied vector
// (p, or r') over the column window the CTA's rows reach, formed while it is
// loaded, and the row sums read shared memory only; in the gather form
// (windows too large) the row sums gather the vector entries and form them
// per nonzero; in the stream form (rows too large for shared memory, the
// window not) the vector is staged as in the window form and the rows are
// read from global memory (L2) in every step. The arithmetic of every row is
// the graph form's (same products, same order of additions, same FP32 / FP64
// rounding points); only the FP64 sums of the per-CTA partials group
// differently. Every CTA sums all partials itself in one fixed order, so all
// CTAs take the same decisions from the same bits and reach the same
// barriers.
//
// The host picks the window form when its footprint fits, else the gather
// form, else the stream form (plan_rows).
//
// Safety: the launch is cooperative (the runtime refuses a grid that cannot
// be co-resident); rows are assigned by blockIdx (no SM ids); every barrier
// wait is bounded and a timeout raises an abort word that releases every
// other waiter; the host checks the per-CTA shared-memory footprint before
// choosing this form.
#include <algorithm>
#include <climits>
#include <vector>

#include "handles.hpp"

namespace mps {
namespace {

constexpr int kPNT = 1024;                       // threads per CTA
constexpr size_t kPSmemBudget = 200 * 1024;      // matrix rows per CTA (dynamic shared memory)
constexpr size_t kPSmemWinBudget = 220 * 1024;   // window form: rows, vector window, own x and D^-1
constexpr unsigned kGridSpinLimit = 1u << 22;    // polls of one barrier wait (about a second)
constexpr int kCountWord = 0;                    // barrier words: [0] arrivals (monotonic),
constexpr int kAbortWord = 2;                    // [2] abort
constexpr int kBarWords = 3;
// Persistent forms: rows in shared memory with the vector gathered per
// nonzero (gather), rows in shared memory with the vector's window staged
// (window), rows read from global memory with the window staged (stream).
constexpr int kGatherForm = 0, kWindowForm = 1, kStreamForm = 2;

struct PersistDev {
    const int* a_rp;
    const int* a_ci;
    const float* a_v;
    const int* m_rp;
    const int* m_ci;
    const float* m_v;
    const int* row_start;   // gridDim.x + 1 row boundaries
    const int* win;         // per CTA [lo, hi): the columns its rows of A and M reach
    const float* dinv;      // Jacobi diagonal (fallback, and the r.D^-1 r sums)
    const double* b;        // FP64 right-hand side
    double* x;              // FP64 solution
    float* r0;              // residual pair (current one by iteration parity)
    float* r1;
    float* p0;              // direction pair
    float* p1;
    float* q;
    float* z;
    double* part;           // partial sums: 4 slots x 3 sums x gridDim.x
    unsigned* bar;          // [0] arrivals (monotonic), [1] unused, [2] abort (zeroed before launch)
    unsigned* err;
    DevScalars* sc_out;     // the final scalars (read back by the host)
    const SolveParams* prm;
    int n;
    const float* b32;       // CG form: FP32 right-hand side
    float* x32;             // CG form: FP32 solution
    const unsigned short* a_c16;   // stream form: A's / M's columns, 16-bit, relative to
    const unsigned short* m_c16;   // the column window of the CTA that owns the row
    unsigned spin_limit;    // polls of one barrier wait before it gives up
    int silent_cta;         // test hook: this CTA skips its first arrival (-1: none)
};

struct PersistShared {
    DevScalars S;                 // this CTA's copy of the solver scalars
    double red[3 * (kPNT / 32)];
    double tot[3];
    unsigned gen;
    int ok;
};

// Vectors that other CTAs of the same launch write (p, q, r, z, x): plain
// weak loads, cached in L1.  Every such read follows a grid barrier
// (reduce_all): the writers' stores precede their CTA's release (bar.sync,
// then thread 0's release add on the counter), and the reader's warp 0
// acquires the counter before the bar.sync that releases its CTA, so by the
// PTX memory model the weak loads observe those stores; within one step no
// CTA writes a vector it gathers.
template <class T>
__device__ __forceinline__ T ldv(const T* p) {
    return *p;
}

__device__ __forceinline__ unsigned ld_volatile_u32(const unsigned* p) {
    return *reinterpret_cast<const volatile unsigned*>(p);
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide FP64 sums of NS per-thread values, fused with the grid barrier.
//   1. block sums (warp butterflies, then warp 0 over the warp totals);
//   2. thread 0 stores the CTA's NS totals in partial slot `slot` and arrives
//      on the grid's monotonic counter with a release add (no return value
//      to wait for); reduction k (k = 1, 2, ...) is complete once the
//      counter reaches k * gridDim.x (compared by signed difference: the
//      counter may wrap);
//   3. warp 0 polls the counter with acquire loads (one address: one request
//      per poll for the warp) and then sums all CTAs' partials -- lane l the
//      partials l, l + 32, ..., then a butterfly -- so every CTA adds the same
//      partials in the same order and gets the same bits;
//   4. thread 0 applies `fin` to the totals (the solver's scalar update), and
//      one bar.sync hands both to the CTA.
// Consecutive reductions must use different slots: a CTA may store its next
// partials while a slower CTA still reads these.  The wait is bounded
// (P.spin_limit polls, back-off after 64); a timeout raises the error word
// and the abort word, and the abort word ends every other CTA's wait.  (The
// test hook P.silent_cta withholds one CTA's first arrival, so every wait of
// that reduction runs out this way.)
// false: this CTA gave up (timeout or abort).
struct NoFin {
    __device__ void operator()(const double*) const {}
};

template <int NS, class Fin = NoFin>
__device__ bool reduce_all(const PersistDev& P, PersistShared& sh, int slot, double (&acc)[NS],
                           double (&tot)[NS], Fin fin = Fin{}) {
    constexpr int W = kPNT / 32;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < NS; ++j) acc[j] = warp_sum(acc[j]);
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < NS; ++j) sh.red[j * W + w] = acc[j];
    }
    __syncthreads();
    if (w == 0) {
        const int G = gridDim.x;
        const unsigned target = (sh.gen + 1) * (unsigned)G;
        double bt[NS];
#pragma unroll
        for (int j = 0; j < NS; ++j) bt[j] = warp_sum(lane < W ? sh.red[j * W + lane] : 0.0);
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < NS; ++j) P.part[(slot * 3 + j) * G + blockIdx.x] = bt[j];
            if (P.silent_cta != (int)blockIdx.x || sh.gen != 0) red_release_add(P.bar + kCountWord, 1u);
        }
        __syncwarp();
        int ok = 1;
        unsigned spins = 0;
        while ((int)(ld_acquire_u32(P.bar + kCountWord) - target) < 0) {
            if (ld_volatile_u32(P.bar + kAbortWord)) {
                ok = 0;
                break;
            }
            if (++spins > P.spin_limit) {
                if (lane == 0) {
                    atomicOr(P.err, kErrTimeout);
                    atomicExch(P.bar + kAbortWord, 1u);
                }
                ok = 0;
                break;
            }
            if (spins > 64) __nanosleep(128);
        }
        ok = __all_sync(0xffffffffu, ok);
        if (ok) {
            // all of a lane's partials are loaded before any is added (one
            // L2 round trip, not one per partial); added in CTA order
            constexpr int U = 5;   // 5 * 32 = 160 CTAs per round
            double s[NS];
#pragma unroll
            for (int j = 0; j < NS; ++j) s[j] = 0.0;
            for (int c0 = lane; c0 < G; c0 += 32 * U) {
                double v[U][NS];
#pragma unroll
                for (int u = 0; u < U; ++u) {
#pragma unroll
                    for (int j = 0; j < NS; ++j)
                        v[u][j] = c0 + 32 * u < G ? __ldcg(P.part + (slot * 3 + j) * G + c0 + 32 * u) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (c0 + 32 * u < G) {
#pragma unroll
                        for (int j = 0; j < NS; ++j) s[j] += v[u][j];
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < NS; ++j) s[j] = warp_sum(s[j]);
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < NS; ++j) sh.tot[j] = s[j];
                fin(s);   // scalar updates from the totals, before the bar.sync
            }
        }
        if (lane == 0) {
            sh.gen = sh.gen + 1;
            sh.ok = ok;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NS; ++j) tot[j] = sh.tot[j];
    return sh.ok != 0;
}

// win[k - lo] = f(k) for k in [lo, hi): each thread loads up to four
// entries before it stores any, so their global loads are in flight
// together (a window is about three entries per thread).
template <class F>
__device__ __forceinline__ void fill_window(float* win, int lo, int hi, F f) {
    for (int k0 = lo + (int)threadIdx.x; k0 < hi; k0 += 4 * kPNT) {
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = k0 + u * kPNT < hi ? f(k0 + u * kPNT) : 0.f;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k0 + u * kPNT < hi) win[k0 + u * kPNT - lo] = v[u];
    }
}

// Byte offset rounded up to a multiple of a (shared-memory layout; the
// pointers are then formed from the shared array itself, so the compiler
// keeps shared-memory addressing for every access through them).
__device__ __forceinline__ size_t round_up(size_t off, size_t a) { return (off + (a - 1)) & ~(a - 1); }

// Column indices in shared memory: the global 32-bit index, or (NARROW)
// 16 bits relative to the window's first column (windows of at most 65,536
// columns).
template <bool NARROW>
using ColIdx = std::conditional_t<NARROW, unsigned short, int>;

// A matrix entry: from shared memory, or (G) a read-only load from global
// memory (the stream form's rows, unchanged for the kernel's lifetime).
template <bool G, class T>
__device__ __forceinline__ T ldm(const T* p) {
    if constexpr (G) return __ldg(p);
    else return *p;
}

// Row li of a block of a CSR (row pointers in shared memory; columns and
// values in shared memory, or G: in global memory) times a gathered vector:
// the products rounded to FP32 first, then added in column order (the tile
// kernels' arithmetic).
template <bool G = false, class IT, class F>
__device__ __forceinline__ float row_f32(const int* rp, const IT* ci, const float* v, int li, F gather) {
    float s = 0.f;
    const int e = rp[li + 1];
    for (int k = rp[li]; k < e; ++k) s = __fadd_rn(s, __fmul_rn(ldm<G>(v + k), gather((int)ldm<G>(ci + k))));
    return s;
}

// Rows li0 and (when has1) li1 at once, each summed in its own column
// order exactly as row_f32 does: the gathers of both rows are issued four at
// a time before their products are added, so the two rows' gather latencies
// overlap instead of adding up.
template <bool G = false, class IT, class F>
__device__ __forceinline__ void row_pair_f32(const int* rp, const IT* ci, const float* v, int li0,
                                             int li1, bool has1, F gather, float& s0, float& s1) {
    const int b0 = rp[li0], e0 = rp[li0 + 1];
    const int b1 = has1 ? rp[li1] : 0, e1 = has1 ? rp[li1 + 1] : 0;
    s0 = 0.f;
    s1 = 0.f;
    const int len = max(e0 - b0, e1 - b1);
    for (int k = 0; k < len; k += 4) {
        float g0[4], g1[4], w0[4], w1[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const bool in0 = b0 + k + u < e0, in1 = b1 + k + u < e1;
            w0[u] = in0 ? ldm<G>(v + b0 + k + u) : 0.f;
            w1[u] = in1 ? ldm<G>(v + b1 + k + u) : 0.f;
            g0[u] = in0 ? gather((int)ldm<G>(ci + b0 + k + u)) : 0.f;
            g1[u] = in1 ? gather((int)ldm<G>(ci + b1 + k + u)) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (b0 + k + u < e0) s0 = __fadd_rn(s0, __fmul_rn(w0[u], g0[u]));
            if (b1 + k + u < e1) s1 = __fadd_rn(s1, __fmul_rn(w1[u], g1[u]));
        }
    }
}

// FORM: kGatherForm, kWindowForm or kStreamForm (see their definition).
template <int FORM>
__global__ void __launch_bounds__(kPNT, 1) fsai_pcg_persistent(PersistDev P) {
    constexpr bool WIN = FORM != kGatherForm;
    constexpr bool STREAM = FORM == kStreamForm;
    extern __shared__ __align__(16) unsigned char psmem[];
    __shared__ PersistShared sh;
    const int tid = threadIdx.x;
    const int r0 = P.row_start[blockIdx.x], r1 = P.row_start[blockIdx.x + 1];
    const int R = r1 - r0;
    const int a0 = P.a_rp[r0], na = P.a_rp[r1] - a0;
    const int m0 = P.m_rp[r0], nm = P.m_rp[r1] - m0;
    // WIN: the multiplied vector over the CTA's column window, staged once
    // per step (coalesced loads) so the row sums read shared memory only
    // for the vector; the own rows' x (FP64, written through to global) and
    // D^-1 stay in shared memory too.  Rows of A and M: in shared memory, or
    // (stream form) only their row pointers, the columns and values read from
    // global memory in every step; in both WIN forms columns are 16-bit,
    // relative to the window.
    // shared layout: arp[R+1] | mrp[R+1] | [aci[na] | mci[nm] | pad | av[na] |
    //                mv[nm] | pad] | (WIN: xs[R] | ds[R] | win[hi - lo])
    using CI = ColIdx<WIN>;
    const int wlo = WIN ? P.win[2 * blockIdx.x] : 0, whi = WIN ? P.win[2 * blockIdx.x + 1] : 0;
    const int coff = wlo;   // global column = coff + stored index (wlo = 0 in the gather form)
    const int* arp;
    const int* mrp;
    const CI* aci;
    const CI* mci;
    const float* av;
    const float* mv;
    size_t off_own = 0;
    if constexpr (STREAM) {
        // row pointers in shared memory (absolute offsets into the global
        // columns and values, so a row's loads need no dependent global load)
        int* arp_s = reinterpret_cast<int*>(psmem);
        int* mrp_s = arp_s + (R + 1);
        for (int i = tid; i <= R; i += kPNT) {
            arp_s[i] = P.a_rp[r0 + i];
            mrp_s[i] = P.m_rp[r0 + i];
        }
        off_own = round_up(8 * (size_t)(R + 1), 8);
        arp = arp_s;
        mrp = mrp_s;
        aci = P.a_c16;
        mci = P.m_c16;
        av = P.a_v;
        mv = P.m_v;
    } else {
        int* arp_s = reinterpret_cast<int*>(psmem);
        int* mrp_s = arp_s + (R + 1);
        CI* aci_s = reinterpret_cast<CI*>(mrp_s + (R + 1));
        CI* mci_s = aci_s + na;
        const size_t off_v = round_up(8 * (size_t)(R + 1) + sizeof(CI) * (size_t)(na + nm), 4);
        float* av_s = reinterpret_cast<float*>(psmem + off_v);
        float* mv_s = av_s + na;
        off_own = round_up(off_v + 4 * (size_t)(na + nm), 8);
        for (int i = tid; i <= R; i += kPNT) {
            arp_s[i] = P.a_rp[r0 + i] - a0;
            mrp_s[i] = P.m_rp[r0 + i] - m0;
        }
        for (int k = tid; k < na; k += kPNT) {
            aci_s[k] = (CI)(P.a_ci[a0 + k] - coff);
            av_s[k] = P.a_v[a0 + k];
        }
        for (int k = tid; k < nm; k += kPNT) {
            mci_s[k] = (CI)(P.m_ci[m0 + k] - coff);
            mv_s[k] = P.m_v[m0 + k];
        }
        arp = arp_s;
        mrp = mrp_s;
        aci = aci_s;
        mci = mci_s;
        av = av_s;
        mv = mv_s;
    }
    double* xs = reinterpret_cast<double*>(psmem + off_own);
    float* ds = reinterpret_cast<float*>(xs + (WIN ? R : 0));
    float* win = ds + (WIN ? R : 0);
    auto wg = [&](int c) { return win[c]; };
    if constexpr (WIN) {
        for (int li = tid; li < R; li += kPNT) {
            xs[li] = 0.0;
            ds[li] = P.dinv[r0 + li];
        }
    }
    if (tid == 0) {
        sh.gen = 0;
        sh.ok = 1;
        sh.S = DevScalars{};
    }
    __syncthreads();
    DevScalars& S = sh.S;
    const Ctx cx{&sh.S, nullptr, nullptr, {}, 0, {}};
    const float* dinv = P.dinv;

    // ---- start: x = 0, r = (float)b; ||b||^2 -----------------------------
    const int mode0 = P.prm->precond;
    {
        double acc[2] = {0.0, 0.0};
        for (int li = tid; li < R; li += kPNT) {
            const int i = r0 + li;
            const double bd = __ldg(P.b + i);
            const float bf = (float)bd;
            P.x[i] = 0.0;
            P.r0[i] = bf;
            if (mode0 == 1) {
                const float zz = bf * dinv[i];
                acc[1] += (double)bf * bf * dinv[i];
                P.p0[i] = zz;
            }
            acc[0] += bd * bd;
        }
        // slot 3: consecutive reductions never share a slot (with Jacobi the
        // first p.q goes to slot 0 while late CTAs may still read this one)
        double tot[2];
        if (!reduce_all<2>(P, sh, 3, acc, tot)) goto out;
        if (tid == 0) cg_init_scalars(cx, P.prm, P.n, mode0, tot[0], tot[1]);
        __syncthreads();
    }
    // z = M r, r.z -> the first direction (fsai_beta restarts it)
    if (!S.done && S.mode == 2) {
        double acc[1] = {0.0};
        const float* rc = P.r0;
        for (int li = tid; li < R; li += kPNT) {
            const float s = row_f32<STREAM>(mrp, mci, mv, li, [&](int c) { return ldv(rc + coff + c); });
            const int i = r0 + li;
            P.z[i] = s;
            acc[0] += (double)ldv(rc + i) * (double)s;
        }
        double tot[1];
        if (!reduce_all<1>(P, sh, 1, acc, tot)) goto out;
        if (tid == 0) fsai_beta(&S, tot[0]);
        __syncthreads();
    }

    while (!S.done) {
        if (!S.replace) {
            // ---- step 1: p = z + beta p_old on the fly, q = A p, p.q -------
            {
                const bool odd = S.iter & 1;
                float* pn = odd ? P.p1 : P.p0;
                const float* po = odd ? P.p0 : P.p1;
                const float* rc = odd ? P.r1 : P.r0;
                const float beta = (float)S.beta;
                const bool jac = S.mode == 1;
                auto dir = [&](int c) {
                    const float zc = jac ? ldv(rc + c) * __ldg(dinv + c) : ldv(P.z + c);
                    return beta != 0.f ? fmaf(beta, ldv(po + c), zc) : zc;
                };
                double acc[1] = {0.0};
                if constexpr (WIN) {
                    fill_window(win, wlo, whi, dir);
                    __syncthreads();
                }
                auto own = [&](int li, float s) {
                    const int i = r0 + li;
                    const float pv = WIN ? win[i - wlo] : dir(i);
                    pn[i] = pv;
                    P.q[i] = s;
                    acc[0] += (double)pv * (double)s;
                };
                for (int li = tid; li < R; li += 2 * kPNT) {
                    const int lj = li + kPNT;
                    const bool has1 = lj < R;
                    float s0, s1;
                    if constexpr (WIN) row_pair_f32<STREAM>(arp, aci, av, li, lj, has1, wg, s0, s1);
                    else row_pair_f32(arp, aci, av, li, lj, has1, dir, s0, s1);
                    own(li, s0);
                    if (has1) own(lj, s1);
                }
                double tot[1];
                if (!reduce_all<1>(P, sh, 0, acc, tot, [&](const double* t) {
                        const double pq = t[0];
                        S.pq = pq;
                        if (!(pq > 0.0) || !isfinite(pq)) {
                            S.breakdown = 1;
                            S.done = 1;
                            S.alpha = 0.0;
                        } else {
                            S.alpha = S.rz / pq;
                        }
                    }))
                    goto out;
                if (S.done) break;
                if constexpr (WIN) {
                    // x += alpha p (FP64) while the window still holds p
                    const double a = S.alpha;
                    for (int li = tid; li < R; li += kPNT) {
                        const double xv = fma(a, (double)win[r0 + li - wlo], xs[li]);
                        xs[li] = xv;
                        P.x[r0 + li] = xv;
                    }
                    // step 2 restages the window (r' over p): every thread's
                    // reads of p above come first
                    __syncthreads();
                }
            }
            // ---- step 2: r' = r - alpha q on the fly, z = M r', x += alpha p
            {
                const bool odd = S.iter & 1;
                const float* rc = odd ? P.r1 : P.r0;
                float* rn = odd ? P.r0 : P.r1;
                const float* pc = odd ? P.p1 : P.p0;
                const double a = S.alpha;
                const float af = (float)a;
                auto res = [&](int c) { return fmaf(-af, ldv(P.q + c), ldv(rc + c)); };
                double acc[3] = {0.0, 0.0, 0.0};
                if constexpr (WIN) {
                    fill_window(win, wlo, whi, res);
                    __syncthreads();
                }
                auto own = [&](int li, float s) {
                    const int i = r0 + li;
                    const float rv = WIN ? win[i - wlo] : res(i);
                    rn[i] = rv;
                    if constexpr (!WIN) P.x[i] = fma(a, (double)ldv(pc + i), ldv(P.x + i));
                    P.z[i] = s;
                    acc[0] += (double)rv * rv;
                    acc[1] += (double)rv * rv * (WIN ? ds[li] : dinv[i]);
                    acc[2] += (double)rv * (double)s;
                };
                for (int li = tid; li < R; li += 2 * kPNT) {
                    const int lj = li + kPNT;
                    const bool has1 = lj < R;
                    float s0, s1;
                    if constexpr (WIN) row_pair_f32<STREAM>(mrp, mci, mv, li, lj, has1, wg, s0, s1);
                    else row_pair_f32(mrp, mci, mv, li, lj, has1, res, s0, s1);
                    own(li, s0);
                    if (has1) own(lj, s1);
                }
                double tot[3];
                if (!reduce_all<3>(P, sh, 1, acc, tot, [&](const double* t) {
                        cg_finalize_ir(&S, t[0], t[1]);
                        if (!S.replace && !S.done && S.mode == 2) fsai_beta(&S, t[2]);
                    }))
                    goto out;
            }
        } else {
            // ---- replacement: r = (float)(b - A x) in FP64 ------------------
            {
                float* rw = (S.iter & 1) ? P.r1 : P.r0;
                double acc[2] = {0.0, 0.0};
                for (int li = tid; li < R; li += kPNT) {
                    double s = 0.0;
                    const int e = arp[li + 1];
                    for (int k = arp[li]; k < e; ++k)
                        s = __dadd_rn(s, __dmul_rn((double)av[k], ldv(P.x + coff + aci[k])));
                    const int i = r0 + li;
                    const double rt = __ldg(P.b + i) - s;
                    const float rf = (float)rt;
                    rw[i] = rf;
                    acc[0] += rt * rt;
                    acc[1] += (double)rf * rf * dinv[i];
                }
                double tot[2];
                if (!reduce_all<2>(P, sh, 2, acc, tot)) goto out;
                if (tid == 0) {
                    S.replace = 0;
                    ++S.replaced;
                    const double rr = tot[0];
                    S.rr = rr;
                    S.rr_ref = rr;
                    if (!isfinite(rr)) {
                        S.breakdown = 1;
                        S.done = 1;
                    } else if (rr <= S.tol2) {
                        S.converged = 1;
                        S.done = 1;
                    } else if (S.iter >= S.max_iter) {
                        S.done = 1;
                    } else {
                        cg_direction(&S, rr, tot[1]);
                        if (S.mode == 2) S.refresh = 1;
                    }
                }
                __syncthreads();
            }
            // z = M r of the replaced residual
            if (!S.done && S.mode == 2 && S.refresh) {
                const float* rc = (S.iter & 1) ? P.r1 : P.r0;
                double acc[1] = {0.0};
                for (int li = tid; li < R; li += kPNT) {
                    const float s = row_f32<STREAM>(mrp, mci, mv, li, [&](int c) { return ldv(rc + coff + c); });
                    const int i = r0 + li;
                    P.z[i] = s;
                    acc[0] += (double)ldv(rc + i) * (double)s;
                }
                double tot[1];
                if (!reduce_all<1>(P, sh, 3, acc, tot)) goto out;
                if (tid == 0) {
                    S.refresh = 0;
                    fsai_beta(&S, tot[0]);
                }
                __syncthreads();
            }
        }
    }
out:
    if (tid == 0 && blockIdx.x == 0) {
        if (!sh.ok) S.err |= kErrTimeout;
        *P.sc_out = S;
    }
}


// Plain CG and Jacobi-PCG (FP32 x and vectors: the drop-in cgd) as one
// cooperative kernel over A's rows held in shared memory.  Per iteration:
//   step 1  p = z + beta p_old on the fly (z = r, or D^-1 r), q = A p, p.q  -> alpha
//   step 2  x += alpha p, r -= alpha q, r.r (and r.D^-1 r)                  -> beta, stop
// with the per-element arithmetic of the graph form's three kernels
// (EpiCgPq, cg_update_xr, cg_update_p) and its stop rule (cg_finalize_xr).
// IR (reliable updates, cg_mixed without FSAI): x accumulated in FP64
// (P.x), b in FP64 (P.b), the stop rule of cg_finalize_ir, and -- when due --
// the residual replacement r = (float)(b - A x) in FP64 in the same kernel.
template <bool IR, int FORM>
__global__ void __launch_bounds__(kPNT, 1) cg_persistent(PersistDev P) {
    constexpr bool WIN = FORM != kGatherForm;
    constexpr bool STREAM = FORM == kStreamForm;
    extern __shared__ __align__(16) unsigned char psmem[];
    __shared__ PersistShared sh;
    const int tid = threadIdx.x;
    const int r0 = P.row_start[blockIdx.x], r1 = P.row_start[blockIdx.x + 1];
    const int R = r1 - r0;
    const int a0 = P.a_rp[r0], na = P.a_rp[r1] - a0;
    // shared layout: arp[R+1] | [aci[na] | pad | av[na]] | pad to 8 (the
    // bracket not in the stream form, whose columns and values are read from
    // global memory); the window and stream forms add the own rows' x (FP64 under IR, written through
    // to global), r (written through), q and D^-1, then the vector window
    // (columns 16-bit, relative to the window, in both forms):
    //   ... | xs[R] | rs[R] | qs[R] | ds[R] | win[hi - lo]
    using XT = std::conditional_t<IR, double, float>;
    using CI = ColIdx<WIN>;   // WIN forms: 16-bit columns relative to the window
    const int wlo = WIN ? P.win[2 * blockIdx.x] : 0, whi = WIN ? P.win[2 * blockIdx.x + 1] : 0;
    const int coff = wlo;   // global column = coff + stored index (wlo = 0 in the gather form)
    const int* arp;
    const CI* aci;
    const float* av;
    size_t off_own = 0;
    if constexpr (STREAM) {
        // row pointers in shared memory (absolute offsets into the global
        // columns and values)
        int* arp_s = reinterpret_cast<int*>(psmem);
        for (int i = tid; i <= R; i += kPNT) arp_s[i] = P.a_rp[r0 + i];
        off_own = round_up(4 * (size_t)(R + 1), 8);
        arp = arp_s;
        aci = P.a_c16;
        av = P.a_v;
    } else {
        int* arp_s = reinterpret_cast<int*>(psmem);
        CI* aci_s = reinterpret_cast<CI*>(arp_s + (R + 1));
        const size_t off_v = round_up(4 * (size_t)(R + 1) + sizeof(CI) * (size_t)na, 4);
        float* av_s = reinterpret_cast<float*>(psmem + off_v);
        off_own = round_up(off_v + 4 * (size_t)na, 8);
        for (int i = tid; i <= R; i += kPNT) arp_s[i] = P.a_rp[r0 + i] - a0;
        for (int k = tid; k < na; k += kPNT) {
            aci_s[k] = (CI)(P.a_ci[a0 + k] - coff);
            av_s[k] = P.a_v[a0 + k];
        }
        arp = arp_s;
        aci = aci_s;
        av = av_s;
    }
    XT* xs = reinterpret_cast<XT*>(psmem + off_own);
    float* rs = reinterpret_cast<float*>(xs + (WIN ? R : 0));
    float* qs = rs + (WIN ? R : 0);
    float* ds = qs + (WIN ? R : 0);
    float* win = ds + (WIN ? R : 0);
    auto wg = [&](int c) { return win[c]; };
    if (tid == 0) {
        sh.gen = 0;
        sh.ok = 1;
        sh.S = DevScalars{};
    }
    __syncthreads();
    DevScalars& S = sh.S;
    const Ctx cx{&sh.S, nullptr, nullptr, {}, 0, {}};
    const int mode0 = P.prm->precond;            // 0 none, 1 Jacobi
    const float* dinv = mode0 == 1 ? P.dinv : nullptr;
    float* r = P.r0;
    if constexpr (WIN) {
        for (int li = tid; li < R; li += kPNT) ds[li] = dinv ? dinv[r0 + li] : 1.f;
    }
    {
        // x = 0, r = b; b.b and b.D^-1 b
        double acc[2] = {0.0, 0.0};
        for (int li = tid; li < R; li += kPNT) {
            const int i = r0 + li;
            if constexpr (IR) {
                const double bd = __ldg(P.b + i);
                const float bf = (float)bd;
                P.x[i] = 0.0;
                r[i] = bf;
                if constexpr (WIN) {
                    xs[li] = 0.0;
                    rs[li] = bf;
                }
                if (dinv) acc[1] += (double)bf * bf * dinv[i];
                acc[0] += bd * bd;
            } else {
                const float bf = P.b32[i];
                P.x32[i] = 0.f;
                r[i] = bf;
                if constexpr (WIN) {
                    xs[li] = 0.f;
                    rs[li] = bf;
                }
                if (dinv) acc[1] += (double)bf * bf * dinv[i];
                acc[0] += (double)bf * bf;
            }
        }
        // slot 3: consecutive reductions never share a slot (the first
        // iteration's p.q goes to slot 0 while late CTAs may still read
        // this one)
        double tot[2];
        if (!reduce_all<2>(P, sh, 3, acc, tot)) goto out;
        if (tid == 0) cg_init_scalars(cx, P.prm, P.n, mode0, tot[0], tot[1]);
        __syncthreads();
    }
    while (!S.done) {
        if (IR && S.replace) {
            // ---- replacement: r = (float)(b - A x) in FP64 ------------------
            double acc[2] = {0.0, 0.0};
            for (int li = tid; li < R; li += kPNT) {
                double sd = 0.0;
                const int e = arp[li + 1];
                for (int k = arp[li]; k < e; ++k)
                    sd = __dadd_rn(sd, __dmul_rn((double)av[k], ldv(P.x + coff + aci[k])));
                const int i = r0 + li;
                const double rt = __ldg(P.b + i) - sd;
                const float rf = (float)rt;
                r[i] = rf;
                if constexpr (WIN) rs[li] = rf;
                acc[0] += rt * rt;
                acc[1] += (double)rf * rf * (dinv ? dinv[i] : 1.f);
            }
            double tot[2];
            if (!reduce_all<2>(P, sh, 2, acc, tot)) goto out;
            if (tid == 0) {
                S.replace = 0;
                ++S.replaced;
                const double rr = tot[0];
                S.rr = rr;
                S.rr_ref = rr;
                if (!isfinite(rr)) {
                    S.breakdown = 1;
                    S.done = 1;
                } else if (rr <= S.tol2) {
                    S.converged = 1;
                    S.done = 1;
                } else if (S.iter >= S.max_iter) {
                    S.done = 1;
                } else {
                    cg_direction(&S, rr, tot[1]);
                }
            }
            __syncthreads();
            continue;
        }
        // ---- step 1: p = z + beta p_old on the fly, q = A p, p.q ----------
        {
            const bool odd = S.iter & 1;
            float* pn = odd ? P.p1 : P.p0;
            const float* po = odd ? P.p0 : P.p1;
            const float beta = (float)S.beta;
            const bool jac = S.mode == 1;
            auto dir = [&](int c) {
                const float zc = jac ? ldv(r + c) * __ldg(P.dinv + c) : ldv(r + c);
                return beta != 0.f ? fmaf(beta, ldv(po + c), zc) : zc;
            };
            double acc[1] = {0.0};
            if constexpr (WIN) {
                fill_window(win, wlo, whi, dir);
                __syncthreads();
            }
            auto own = [&](int li, float sv) {
                const int i = r0 + li;
                const float pv = WIN ? win[i - wlo] : dir(i);
                pn[i] = pv;
                if constexpr (WIN) qs[li] = sv;
                else P.q[i] = sv;
                acc[0] += (double)pv * (double)sv;
            };
            for (int li = tid; li < R; li += 2 * kPNT) {
                const int lj = li + kPNT;
                const bool has1 = lj < R;
                float s0, s1;
                if constexpr (WIN) row_pair_f32<STREAM>(arp, aci, av, li, lj, has1, wg, s0, s1);
                else row_pair_f32(arp, aci, av, li, lj, has1, dir, s0, s1);
                own(li, s0);
                if (has1) own(lj, s1);
            }
            double tot[1];
            if (!reduce_all<1>(P, sh, 0, acc, tot, [&](const double* t) {
                    const double pq = t[0];
                    S.pq = pq;
                    if (!(pq > 0.0) || !isfinite(pq)) {
                        S.breakdown = 1;
                        S.done = 1;
                        S.alpha = 0.0;
                    } else {
                        S.alpha = S.rz / pq;
                    }
                }))
                goto out;
            if (S.done) break;
        }
        // ---- step 2: x += alpha p, r -= alpha q, r.r, r.D^-1 r -------------
        {
            const float* pc = (S.iter & 1) ? P.p1 : P.p0;
            const double a64 = S.alpha;
            const float a = (float)a64;
            double acc[2] = {0.0, 0.0};
            for (int li = tid; li < R; li += kPNT) {
                const int i = r0 + li;
                float rv;
                if constexpr (WIN) {
                    // p is still in the window; x, r, q, D^-1 of own rows in
                    // shared memory (x and r written through)
                    const float pv = win[i - wlo];
                    if constexpr (IR) {
                        const double xv = fma(a64, (double)pv, xs[li]);
                        xs[li] = xv;
                        P.x[i] = xv;
                    } else {
                        const float xv = fmaf(a, pv, xs[li]);
                        xs[li] = xv;
                        P.x32[i] = xv;
                    }
                    rv = fmaf(-a, qs[li], rs[li]);
                    rs[li] = rv;
                    r[i] = rv;
                    acc[0] += (double)rv * rv;
                    if (dinv) acc[1] += (double)rv * rv * ds[li];
                } else {
                    if constexpr (IR) P.x[i] = fma(a64, (double)ldv(pc + i), ldv(P.x + i));
                    else P.x32[i] = fmaf(a, ldv(pc + i), ldv(P.x32 + i));
                    rv = fmaf(-a, ldv(P.q + i), ldv(r + i));
                    r[i] = rv;
                    acc[0] += (double)rv * rv;
                    if (dinv) acc[1] += (double)rv * rv * dinv[i];
                }
            }
            double tot[2];
            if (!reduce_all<2>(P, sh, 1, acc, tot, [&](const double* t) {
                    if constexpr (IR) cg_finalize_ir(&S, t[0], t[1]);
                    else cg_finalize_xr(&S, t[0], t[1]);
                }))
                goto out;
        }
    }
out:
    if (tid == 0 && blockIdx.x == 0) {
        if (!sh.ok) S.err |= kErrTimeout;
        *P.sc_out = S;
    }
}

// BiCGSTAB (the drop-in bicgstab, outside reference_compat) as one
// cooperative kernel over A's rows held in shared memory.  Per iteration,
// each step separated from the next by a grid-wide sum:
//   A  p = r + beta (p_old - omega v_old) (first iteration: p = r), formed
//      while staging it; v = A p; sigma = r0.v                -> alpha
//   B  s = r - alpha v, formed while staging it; t = A s;
//      t.s, t.t                                               -> omega
//   C  x += alpha p + omega s; r = s - omega t; r0.r, r.r     -> beta, stop
// with the graph form's per-element arithmetic (bicg_update_p, EpiBicgV,
// bicg_update_s, EpiBicgT, bicg_update_xr) and its stop rule
// (bicg_stop_beta).  p and v are double-buffered by iteration parity: a CTA
// writes its rows of the new ones while slower CTAs still gather the old.
// s and t are never written to global memory: every CTA forms s over its
// own window (gather form: per gathered nonzero), and keeps its rows of t in
// shared memory.  All three forms (the launch adds the own rows' x and t to
// the gather form's footprint).  Buffers: P.r0 = r, P.r1 = r0 (the shadow residual),
// P.p0 / P.p1 = p, P.q / P.z = v, P.b32 = b, P.x32 = x.
template <int FORM>
__global__ void __launch_bounds__(kPNT, 1) bicg_persistent(PersistDev P) {
    extern __shared__ __align__(16) unsigned char psmem[];
    __shared__ PersistShared sh;
    const int tid = threadIdx.x;
    const int r0 = P.row_start[blockIdx.x], r1 = P.row_start[blockIdx.x + 1];
    const int R = r1 - r0;
    const int a0 = P.a_rp[r0], na = P.a_rp[r1] - a0;
    // shared layout: arp[R+1] | [aci[na] | pad | av[na]] | pad to 8 (the
    // stream form reads its columns and values from global memory; columns
    // 16-bit, window-relative in the window and stream forms) | xs[R] | ts[R]
    // | (WIN: win[hi - lo])
    constexpr bool WIN = FORM != kGatherForm;
    constexpr bool STREAM = FORM == kStreamForm;
    using CI = ColIdx<WIN>;
    const int wlo = WIN ? P.win[2 * blockIdx.x] : 0, whi = WIN ? P.win[2 * blockIdx.x + 1] : 0;
    const int coff = wlo;   // global column = coff + stored index (wlo = 0 in the gather form)
    const int* arp;
    const CI* aci;
    const float* av;
    size_t off_own = 0;
    if constexpr (STREAM) {
        // row pointers in shared memory (absolute offsets into the global
        // columns and values)
        int* arp_s = reinterpret_cast<int*>(psmem);
        for (int i = tid; i <= R; i += kPNT) arp_s[i] = P.a_rp[r0 + i];
        off_own = round_up(4 * (size_t)(R + 1), 8);
        arp = arp_s;
        aci = P.a_c16;
        av = P.a_v;
    } else {
        int* arp_s = reinterpret_cast<int*>(psmem);
        CI* aci_s = reinterpret_cast<CI*>(arp_s + (R + 1));
        const size_t off_v = round_up(4 * (size_t)(R + 1) + sizeof(CI) * (size_t)na, 4);
        float* av_s = reinterpret_cast<float*>(psmem + off_v);
        off_own = round_up(off_v + 4 * (size_t)na, 8);
        for (int i = tid; i <= R; i += kPNT) arp_s[i] = P.a_rp[r0 + i] - a0;
        for (int k = tid; k < na; k += kPNT) {
            aci_s[k] = (CI)(P.a_ci[a0 + k] - coff);
            av_s[k] = P.a_v[a0 + k];
        }
        arp = arp_s;
        aci = aci_s;
        av = av_s;
    }
    float* xs = reinterpret_cast<float*>(psmem + off_own);
    float* ts = xs + R;
    float* win = ts + R;
    auto wg = [&](int c) { return win[c]; };
    if (tid == 0) {
        sh.gen = 0;
        sh.ok = 1;
        sh.S = DevScalars{};
    }
    __syncthreads();
    DevScalars& S = sh.S;
    const Ctx cx{&sh.S, nullptr, nullptr, {}, 0, {}};
    float* r = P.r0;
    float* rh = P.r1;
    {
        // x = 0, r = r0 = b; b.b (bicg_init)
        double acc[1] = {0.0};
        for (int li = tid; li < R; li += kPNT) {
            const int i = r0 + li;
            const float bf = P.b32[i];
            xs[li] = 0.f;
            P.x32[i] = 0.f;
            r[i] = bf;
            rh[i] = bf;
            acc[0] += (double)bf * bf;
        }
        double tot[1];
        if (!reduce_all<1>(P, sh, 3, acc, tot, [&](const double* t) { bicg_init_scalars(cx, P.prm, P.n, t[0]); }))
            goto out;
    }
    while (!S.done) {
        const bool odd = S.iter & 1;
        float* pn = odd ? P.p1 : P.p0;
        const float* po = odd ? P.p0 : P.p1;
        float* vn = odd ? P.z : P.q;
        const float* vo = odd ? P.q : P.z;
        // ---- A: p (staged), v = A p, sigma = r0.v -----------------------
        {
            const bool first = S.iter == 0;
            const float beta = (float)S.beta, omega = (float)S.omega;
            auto dirp = [&](int c) {
                return first ? ldv(r + c) : fmaf(beta, fmaf(-omega, ldv(vo + c), ldv(po + c)), ldv(r + c));
            };
            if constexpr (WIN) {
                fill_window(win, wlo, whi, dirp);
                __syncthreads();
            }
            double acc[1] = {0.0};
            auto own = [&](int li, float s) {
                const int i = r0 + li;
                pn[i] = WIN ? win[i - wlo] : dirp(i);
                vn[i] = s;
                acc[0] += (double)rh[i] * (double)s;
            };
            for (int li = tid; li < R; li += 2 * kPNT) {
                const int lj = li + kPNT;
                const bool has1 = lj < R;
                float s0, s1;
                if constexpr (WIN) row_pair_f32<STREAM>(arp, aci, av, li, lj, has1, wg, s0, s1);
                else row_pair_f32(arp, aci, av, li, lj, has1, dirp, s0, s1);
                own(li, s0);
                if (has1) own(lj, s1);
            }
            double tot[1];
            if (!reduce_all<1>(P, sh, 0, acc, tot, [&](const double* t) {
                    const double sigma = t[0];
                    S.sigma = sigma;
                    if (sigma == 0.0 || !isfinite(sigma)) {   // EpiBicgV outside reference_compat
                        S.breakdown = 1;
                        S.done = 1;
                        S.alpha = 0.0;
                    } else {
                        S.alpha = S.rho / sigma;
                    }
                }))
                goto out;
            if (S.done) break;
        }
        // ---- B: s = r - alpha v (staged), t = A s, t.s, t.t ---------------
        const float af = (float)S.alpha;
        auto dirs = [&](int c) { return fmaf(-af, ldv(vn + c), ldv(r + c)); };
        {
            if constexpr (WIN) {
                fill_window(win, wlo, whi, dirs);
                __syncthreads();
            }
            double acc[2] = {0.0, 0.0};
            auto own = [&](int li, float t) {
                const int i = r0 + li;
                const float sv = WIN ? win[i - wlo] : dirs(i);
                ts[li] = t;
                acc[0] += (double)t * (double)sv;
                acc[1] += (double)t * (double)t;
            };
            for (int li = tid; li < R; li += 2 * kPNT) {
                const int lj = li + kPNT;
                const bool has1 = lj < R;
                float s0, s1;
                if constexpr (WIN) row_pair_f32<STREAM>(arp, aci, av, li, lj, has1, wg, s0, s1);
                else row_pair_f32(arp, aci, av, li, lj, has1, dirs, s0, s1);
                own(li, s0);
                if (has1) own(lj, s1);
            }
            double tot[2];
            if (!reduce_all<2>(P, sh, 1, acc, tot, [&](const double* t) {
                    S.phi1 = t[0];
                    S.phi2 = t[1];
                    S.omega = fabs(t[1]) < 1e-20 ? 0.0 : t[0] / t[1];   // EpiBicgT
                }))
                goto out;
        }
        // ---- C: x += alpha p + omega s, r = s - omega t, r0.r, r.r ---------
        {
            const float w = (float)S.omega;
            double acc[2] = {0.0, 0.0};
            for (int li = tid; li < R; li += kPNT) {
                const int i = r0 + li;
                // s of the own row: from the window, or formed again from r
                // and v (read before this thread overwrites r[i] below)
                const float sv = WIN ? win[i - wlo] : dirs(i);
                float xv = fmaf(af, ldv(pn + i), xs[li]);
                xv = fmaf(w, sv, xv);
                xs[li] = xv;
                P.x32[i] = xv;
                const float rv = fmaf(-w, ts[li], sv);
                r[i] = rv;
                acc[0] += (double)rh[i] * (double)rv;
                acc[1] += (double)rv * (double)rv;
            }
            double tot[2];
            if (!reduce_all<2>(P, sh, 2, acc, tot, [&](const double* t) {
                    S.iter = S.iter + 1;
                    S.rho_old = S.rho;
                    S.rho = t[0];
                    S.rnorm2 = t[1];
                    bicg_stop_beta(&S);
                }))
                goto out;
        }
    }
out:
    if (tid == 0 && blockIdx.x == 0) {
        if (!sh.ok) S.err |= kErrTimeout;
        *P.sc_out = S;
    }
}

// Richardson (the drop-in richardson, outside reference_compat) as one
// cooperative kernel: per iteration the CTA stages x_in over its window (or
// gathers it, gather form), forms its rows' x_out = x_in + (w b + (-w) A x_in)
// with the graph form's arithmetic (rich_update) into the other x buffer,
// and sums ||b - A x_in||^2 for the stop rule (rich_finalize): one grid sum
// per iteration.  x is double-buffered by iteration parity (P.x32 even,
// P.q odd, the graph form's vX / vXAlt), so a CTA writes its rows of x_out
// while slower CTAs still read x_in; the grid sums alternate between slots
// 0 and 1.  x itself does not depend on any sum, so for a given iteration
// count every form returns the graph form's bits.
template <int FORM>
__global__ void __launch_bounds__(kPNT, 1) rich_persistent(PersistDev P) {
    constexpr bool WIN = FORM != kGatherForm;
    constexpr bool STREAM = FORM == kStreamForm;
    extern __shared__ __align__(16) unsigned char psmem[];
    __shared__ PersistShared sh;
    const int tid = threadIdx.x;
    const int r0 = P.row_start[blockIdx.x], r1 = P.row_start[blockIdx.x + 1];
    const int R = r1 - r0;
    const int a0 = P.a_rp[r0], na = P.a_rp[r1] - a0;
    // shared layout: arp[R+1] | [aci[na] | pad | av[na]] | pad to 8 (the
    // bracket not in the stream form) | (WIN: win[hi - lo]); columns 16-bit,
    // window-relative in the window and stream forms
    using CI = ColIdx<WIN>;
    const int wlo = WIN ? P.win[2 * blockIdx.x] : 0, whi = WIN ? P.win[2 * blockIdx.x + 1] : 0;
    const int coff = wlo;   // global column = coff + stored index (wlo = 0 in the gather form)
    const int* arp;
    const CI* aci;
    const float* av;
    size_t off_own = 0;
    if constexpr (STREAM) {
        int* arp_s = reinterpret_cast<int*>(psmem);
        for (int i = tid; i <= R; i += kPNT) arp_s[i] = P.a_rp[r0 + i];
        off_own = round_up(4 * (size_t)(R + 1), 8);
        arp = arp_s;
        aci = P.a_c16;
        av = P.a_v;
    } else {
        int* arp_s = reinterpret_cast<int*>(psmem);
        CI* aci_s = reinterpret_cast<CI*>(arp_s + (R + 1));
        const size_t off_v = round_up(4 * (size_t)(R + 1) + sizeof(CI) * (size_t)na, 4);
        float* av_s = reinterpret_cast<float*>(psmem + off_v);
        off_own = round_up(off_v + 4 * (size_t)na, 8);
        for (int i = tid; i <= R; i += kPNT) arp_s[i] = P.a_rp[r0 + i] - a0;
        for (int k = tid; k < na; k += kPNT) {
            aci_s[k] = (CI)(P.a_ci[a0 + k] - coff);
            av_s[k] = P.a_v[a0 + k];
        }
        arp = arp_s;
        aci = aci_s;
        av = av_s;
    }
    float* win = reinterpret_cast<float*>(psmem + off_own);
    auto wg = [&](int c) { return win[c]; };
    if (tid == 0) {
        sh.gen = 0;
        sh.ok = 1;
        sh.S = DevScalars{};
    }
    __syncthreads();
    DevScalars& S = sh.S;
    {
        // x = 0; ||b||^2 (rich_init)
        double acc[1] = {0.0};
        for (int li = tid; li < R; li += kPNT) {
            const int i = r0 + li;
            const float bv = P.b32[i];
            P.x32[i] = 0.f;
            acc[0] += (double)bv * bv;
        }
        double tot[1];
        if (!reduce_all<1>(P, sh, 3, acc, tot, [&](const double* t) { rich_init_scalars(&S, P.prm, P.n, t[0]); }))
            goto out;
    }
    while (!S.done) {
        const bool odd = S.iter & 1;
        const float* xin = odd ? P.q : P.x32;
        float* xout = odd ? P.x32 : P.q;
        const float w = (float)S.omega_rich;
        auto xg = [&](int c) { return ldv(xin + c); };
        if constexpr (WIN) {
            fill_window(win, wlo, whi, xg);
            __syncthreads();
        }
        double acc[1] = {0.0};
        auto own = [&](int li, float ax) {
            const int i = r0 + li;
            const float bv = P.b32[i];
            const float xv = WIN ? win[i - wlo] : xg(i);
            xout[i] = rich_update(xv, w, bv, ax);
            const double res = (double)bv - (double)ax;
            acc[0] += res * res;
        };
        for (int li = tid; li < R; li += 2 * kPNT) {
            const int lj = li + kPNT;
            const bool has1 = lj < R;
            float s0, s1;
            if constexpr (WIN) row_pair_f32<STREAM>(arp, aci, av, li, lj, has1, wg, s0, s1);
            else row_pair_f32(arp, aci, av, li, lj, has1, xg, s0, s1);
            own(li, s0);
            if (has1) own(lj, s1);
        }
        double tot[1];
        if (!reduce_all<1>(P, sh, odd ? 1 : 0, acc, tot, [&](const double* t) { rich_finalize(&S, t[0]); }))
            goto out;
    }
out:
    if (tid == 0 && blockIdx.x == 0) {
        if (!sh.ok) S.err |= kErrTimeout;
        *P.sc_out = S;
    }
}

// Row blocks for `grid` CTAs balanced by their shared-memory bytes
// (4 * words per row + 8 per nonzero of A, and of M when given): boundary c
// is the first row whose prefix reaches c / grid of the total.  Each
// boundary is its own binary search over the row pointers (the prefix is
// monotone), so the result does not depend on the search order.
__global__ void persist_split_kernel(const int* __restrict__ a_rp, const int* __restrict__ m_rp, int n,
                                     int grid, int words, int* __restrict__ start) {
    auto bytes_to = [&](int i) {   // rows [0, i)
        return 4.0 * words * i + 8.0 * ((double)a_rp[i] + (m_rp ? (double)m_rp[i] : 0.0));
    };
    const double total = bytes_to(n);
    for (int c = threadIdx.x; c <= grid; c += blockDim.x) {
        int a = 0, bnd = n;
        if (c == 0) {
            bnd = 0;
        } else if (c < grid) {
            const double target = total * c / grid;
            while (a < bnd) {   // first row whose prefix reaches the target
                const int mid = a + (bnd - a) / 2;
                if (bytes_to(mid) < target) a = mid + 1;
                else bnd = mid;
            }
        } else {
            a = n;
        }
        start[c] = c == 0 ? 0 : a;
    }
}

// Per CTA block: the smallest column, and one past the largest, that its
// rows of A (and M) reference, widened to the block's own rows -- the window
// of the multiplied vector the block's row sums read.
__global__ void persist_window_kernel(const int* __restrict__ a_rp, const int* __restrict__ a_ci,
                                      const int* __restrict__ m_rp, const int* __restrict__ m_ci,
                                      const int* __restrict__ row_start, int* __restrict__ win,
                                      int* __restrict__ cnt) {
    const int b = blockIdx.x;
    const int r0 = row_start[b], r1 = row_start[b + 1];
    if (threadIdx.x == 0) {   // the block's nonzeros of A and M
        cnt[2 * b] = a_rp[r1] - a_rp[r0];
        cnt[2 * b + 1] = m_rp ? m_rp[r1] - m_rp[r0] : 0;
    }
    int lo = r0, hi = r1;
    for (int k = a_rp[r0] + threadIdx.x; k < a_rp[r1]; k += blockDim.x) {
        const int c = a_ci[k];
        lo = min(lo, c);
        hi = max(hi, c + 1);
    }
    if (m_rp) {
        for (int k = m_rp[r0] + threadIdx.x; k < m_rp[r1]; k += blockDim.x) {
            const int c = m_ci[k];
            lo = min(lo, c);
            hi = max(hi, c + 1);
        }
    }
    __shared__ int s_lo[32], s_hi[32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if (lane == 0) {
        s_lo[w] = lo;
        s_hi[w] = hi;
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        lo = __reduce_min_sync(0xffffffffu, lane < nw ? s_lo[lane] : INT_MAX);
        hi = __reduce_max_sync(0xffffffffu, lane < nw ? s_hi[lane] : INT_MIN);
        if (lane == 0) {
            win[2 * b] = lo;
            win[2 * b + 1] = hi;
        }
    }
}

// Stream form: every nonzero's column relative to the column window of the
// CTA that owns its row (CTA b = block b; windows of at most 65,536 columns).
__global__ void persist_c16_kernel(const int* __restrict__ rp, const int* __restrict__ ci,
                                   const int* __restrict__ row_start, const int* __restrict__ win,
                                   unsigned short* __restrict__ out) {
    const int b = blockIdx.x;
    const int lo = win[2 * b];
    const int e = rp[row_start[b + 1]];
    for (int k = rp[row_start[b]] + (int)threadIdx.x; k < e; k += blockDim.x) out[k] = (unsigned short)(ci[k] - lo);
}

}  // namespace

// Row blocks for one CTA per SM over A's rows (and M's when given), split
// and measured on the GPU (one small read-back), balanced by their
// shared-memory bytes; pp.state = -1 when a block would not fit or the
// kernel cannot be made resident (the graph form runs then).
static cudaError_t plan_rows(PersistPlan& pp, int n, const void* kernel, const CsrMat& A, const CsrMat* M,
                             int pick, cudaStream_t s) {
    pp.state = -1;
    int per_sm = 0;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kPSmemBudget);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPNT, kPSmemBudget);
    if (e != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        return cudaSuccess;   // not eligible
    }
    const int words = M ? 2 : 1;   // row-pointer words per row
    // at least 128 rows per CTA; one CTA per SM at most
    const int grid = std::min(num_sms(), std::max(1, n / 128));
    dev_free(pp.d_row_start);
    pp.d_row_start = nullptr;
    dev_free(pp.d_c16);
    pp.d_c16 = nullptr;
    // grid + 1 boundaries, the barrier words, 2 window bounds per block, then
    // 2 nonzero counts per block (read back here only)
    const size_t words_all = (size_t)grid + 1 + kBarWords + 4 * (size_t)grid;
    e = dev_alloc(&pp.d_row_start, words_all * 4, s);
    if (e != cudaSuccess) return e;
    int* d_win = pp.d_row_start + grid + 1 + kBarWords;
    int* d_cnt = d_win + 2 * grid;
    persist_split_kernel<<<1, 256, 0, s>>>(A.rp, M ? M->rp : nullptr, n, grid, words, pp.d_row_start);
    persist_window_kernel<<<grid, 256, 0, s>>>(A.rp, A.ci, M ? M->rp : nullptr, M ? M->ci : nullptr,
                                               pp.d_row_start, d_win, d_cnt);
    e = cudaGetLastError();
    std::vector<int> h(words_all);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), pp.d_row_start, words_all * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    const int* start = h.data();
    const int* win = start + grid + 1 + kBarWords;
    const int* cnt = win + 2 * grid;
    size_t worst = 0, worst_win = 0, worst_stream = 0;
    int rows_max = 0;
    for (int c = 0; c < grid; ++c) {
        const int rows = start[c + 1] - start[c];
        if (rows < 0) return cudaSuccess;
        rows_max = std::max(rows_max, rows);
        size_t b = 4 * (size_t)words * ((size_t)rows + 1) + 8 * (size_t)cnt[2 * c];
        if (M) b += 8 * (size_t)cnt[2 * c + 1];
        worst = std::max(worst, b);
        // window form: 16-bit window-relative columns (6 bytes per
        // nonzero), the vector window and the own rows' vectors beside the
        // rows, 12 bytes of alignment padding
        const size_t w = (size_t)(win[2 * c + 1] - win[2 * c]);
        const size_t nz = (size_t)cnt[2 * c] + (M ? (size_t)cnt[2 * c + 1] : 0);
        const size_t bw = 4 * (size_t)words * ((size_t)rows + 1) + 6 * nz + 12 + 4 * w +
                          (M ? 12 : 20) * (size_t)rows;   // FSAI: x, D^-1; CG: x, r, q, D^-1
        worst_win = std::max(worst_win, w > 65536 ? ~(size_t)0 : bw);
        // stream form: the row pointers, the vector window and the own rows'
        // vectors (columns stored 16-bit relative to the window, in global
        // memory with the values); 4 bytes of alignment padding
        const size_t bs = 4 * (size_t)words * ((size_t)rows + 1) + 4 + 4 * w + (M ? 12 : 20) * (size_t)rows;
        worst_stream = std::max(worst_stream, w > 65536 ? ~(size_t)0 : bs);
    }
    pp.grid = grid;
    pp.rows_max = rows_max;
    // a footprint above the gather budget must still leave one CTA
    // resident per SM
    auto resident = [&](size_t need) {
        if (need > kPSmemWinBudget) return false;
        const int sz = (int)(((need + 15) / 16) * 16);
        int per = 0;
        cudaError_t ew = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        if (ew == cudaSuccess) ew = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kPNT, sz);
        if (ew != cudaSuccess || per < 1) {
            cudaGetLastError();
            return false;
        }
        return true;
    };
    // pick: 0 the first form that fits (window, gather, stream); 1 + form:
    // that form only
    auto may = [&](int f) { return pick == 0 || pick == 1 + f; };
    size_t need;
    if (may(kWindowForm) && resident(worst_win)) {
        pp.form = kWindowForm;
        need = worst_win;
    } else if (may(kGatherForm) && worst <= kPSmemBudget) {
        pp.form = kGatherForm;
        need = worst;
    } else if (may(kStreamForm) && resident(worst_stream)) {
        pp.form = kStreamForm;
        need = worst_stream;
        // the rows' columns relative to their CTA's window, 16-bit, in
        // global memory (built once per pattern; values are read from the
        // matrix itself)
        const size_t nz = (size_t)A.nnz + (M ? (size_t)M->nnz : 0);
        e = dev_alloc(&pp.d_c16, 2 * nz, s);
        if (e != cudaSuccess) {   // no room: the graph form runs
            cudaGetLastError();
            pp.d_c16 = nullptr;
            return cudaSuccess;
        }
        const int* d_win = pp.d_row_start + grid + 1 + kBarWords;
        persist_c16_kernel<<<grid, 256, 0, s>>>(A.rp, A.ci, pp.d_row_start, d_win, pp.d_c16);
        if (M) persist_c16_kernel<<<grid, 256, 0, s>>>(M->rp, M->ci, pp.d_row_start, d_win, pp.d_c16 + A.nnz);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    } else {
        return cudaSuccess;   // not eligible: the graph form runs
    }
    pp.smem = ((need + 15) / 16) * 16;
    pp.state = 1;
    return cudaSuccess;
}

// Plan of the FSAI form (rows of A and M).
cudaError_t persist_plan_build(mps_csr* h, cudaStream_t s) {
    h->pp.state = -1;
    if (!h->use_m || !h->M.rp || h->A.n_rows != h->M.n_rows) return cudaSuccess;
    return plan_rows(h->pp, (int)h->A.n_rows, reinterpret_cast<const void*>(fsai_pcg_persistent<kGatherForm>),
                     h->A, &h->M, h->persist_form, s);
}

// Plan of the CG form (rows of A only).
cudaError_t persist_plan_build_a(mps_csr* h, cudaStream_t s) {
    h->pp_a.state = -1;
    if (h->A.n_rows != h->A.n_cols) return cudaSuccess;
    return plan_rows(h->pp_a, (int)h->A.n_rows, reinterpret_cast<const void*>(cg_persistent<false, kGatherForm>),
                     h->A, nullptr, h->persist_form, s);
}

// Plain CG / Jacobi-PCG as one cooperative launch: b is H.v(vB), x lands in
// H.v(vX) and the final scalars in H.ws.sc (the graph form's places); with
// b64 / x64 given, the reliable-update form (FP64 b and x, the caller's
// buffers).  The parameters must be in H.ws.d_params.
// cudaErrorNotSupported: A's rows do not fit (the graph form runs then).
cudaError_t persist_cg_solve(mps_csr* h, cudaStream_t s, const double* b64, double* x64) {
    if (h->pp_a.state == 0) {
        const cudaError_t e = persist_plan_build_a(h, s);
        if (e != cudaSuccess) return e;
    }
    if (h->pp_a.state != 1) return cudaErrorNotSupported;
    SolverHost& H = h->H;
    PersistDev P{};
    P.a_rp = h->A.rp;
    P.a_ci = h->A.ci;
    P.a_v = h->A.v;
    P.row_start = h->pp_a.d_row_start;
    P.dinv = H.dinv;
    P.r0 = H.v(vR);
    P.p0 = H.v(vP);
    P.p1 = H.v(vP1);
    P.q = H.v(vQ);
    P.part = H.ws.partials;
    P.bar = reinterpret_cast<unsigned*>(h->pp_a.d_row_start + h->pp_a.grid + 1);
    P.err = h->d_err;
    P.sc_out = H.ws.sc;
    P.prm = H.ws.d_params;
    P.n = (int)h->A.n_rows;
    P.spin_limit = h->test_spin_limit ? h->test_spin_limit : kGridSpinLimit;
    P.silent_cta = h->test_silent_cta;
    P.b32 = H.v(vB);
    P.x32 = H.v(vX);
    P.b = b64;
    P.x = x64;
    P.win = h->pp_a.d_row_start + h->pp_a.grid + 1 + kBarWords;
    P.a_c16 = h->pp_a.d_c16;
    const int f = h->pp_a.form;
    const void* k;
    if (b64)
        k = f == kWindowForm ? reinterpret_cast<const void*>(cg_persistent<true, kWindowForm>)
            : f == kStreamForm ? reinterpret_cast<const void*>(cg_persistent<true, kStreamForm>)
                               : reinterpret_cast<const void*>(cg_persistent<true, kGatherForm>);
    else
        k = f == kWindowForm ? reinterpret_cast<const void*>(cg_persistent<false, kWindowForm>)
            : f == kStreamForm ? reinterpret_cast<const void*>(cg_persistent<false, kStreamForm>)
                               : reinterpret_cast<const void*>(cg_persistent<false, kGatherForm>);
    cudaError_t e = cudaMemsetAsync(P.bar, 0, kBarWords * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->pp_a.smem);
    if (e != cudaSuccess) return e;
    void* args[] = {&P};
    return cudaLaunchCooperativeKernel(k, dim3(h->pp_a.grid), dim3(kPNT), args, h->pp_a.smem, s);
}

// BiCGSTAB as one cooperative launch (any form): b is H.v(vB), x
// lands in H.v(vX) and the final scalars in H.ws.sc; the parameters must be
// in H.ws.d_params.  cudaErrorNotSupported: not eligible (the graph form runs).
cudaError_t persist_bicg_solve(mps_csr* h, cudaStream_t s) {
    if (h->pp_a.state == 0) {
        const cudaError_t e = persist_plan_build_a(h, s);
        if (e != cudaSuccess) return e;
    }
    if (h->pp_a.state != 1) return cudaErrorNotSupported;
    const int f = h->pp_a.form;
    size_t smem = h->pp_a.smem;
    if (f == kGatherForm) {
        // the gather form's footprint holds A's rows only: add the own rows'
        // x and t (and 8 bytes of alignment); it must still fit one CTA per SM
        smem = ((smem + 8 * (size_t)h->pp_a.rows_max + 8 + 15) / 16) * 16;
        const void* kg = reinterpret_cast<const void*>(bicg_persistent<kGatherForm>);
        int per = 0;
        cudaError_t eg = smem <= kPSmemWinBudget ? cudaSuccess : cudaErrorInvalidValue;
        if (eg == cudaSuccess) eg = cudaFuncSetAttribute(kg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (eg == cudaSuccess) eg = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kg, kPNT, smem);
        if (eg != cudaSuccess || per < 1) {
            cudaGetLastError();
            return cudaErrorNotSupported;
        }
    }
    SolverHost& H = h->H;
    PersistDev P{};
    P.a_rp = h->A.rp;
    P.a_ci = h->A.ci;
    P.a_v = h->A.v;
    P.row_start = h->pp_a.d_row_start;
    P.win = h->pp_a.d_row_start + h->pp_a.grid + 1 + kBarWords;
    P.r0 = H.v(vR);
    P.r1 = H.v(vR0);
    P.p0 = H.v(vP);
    P.p1 = H.v(vS);
    P.q = H.v(vQ);
    P.z = H.v(vT);
    P.part = H.ws.partials;
    P.bar = reinterpret_cast<unsigned*>(h->pp_a.d_row_start + h->pp_a.grid + 1);
    P.err = h->d_err;
    P.sc_out = H.ws.sc;
    P.prm = H.ws.d_params;
    P.n = (int)h->A.n_rows;
    P.spin_limit = h->test_spin_limit ? h->test_spin_limit : kGridSpinLimit;
    P.silent_cta = h->test_silent_cta;
    P.b32 = H.v(vB);
    P.x32 = H.v(vX);
    P.a_c16 = h->pp_a.d_c16;
    const void* k = f == kStreamForm   ? reinterpret_cast<const void*>(bicg_persistent<kStreamForm>)
                    : f == kWindowForm ? reinterpret_cast<const void*>(bicg_persistent<kWindowForm>)
                                       : reinterpret_cast<const void*>(bicg_persistent<kGatherForm>);
    cudaError_t e = cudaMemsetAsync(P.bar, 0, kBarWords * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    void* args[] = {&P};
    return cudaLaunchCooperativeKernel(k, dim3(h->pp_a.grid), dim3(kPNT), args, smem, s);
}

// Richardson as one cooperative launch (any form; the CG plan, whose
// own-row budget covers it): b is H.v(vB); x ends in H.v(vX) or H.v(vXAlt)
// by the parity of the final iteration count (as in the graph form:
// copy_result selects it); the final scalars in H.ws.sc, the parameters in
// H.ws.d_params.  cudaErrorNotSupported: not eligible (the graph form runs).
cudaError_t persist_rich_solve(mps_csr* h, cudaStream_t s) {
    if (h->pp_a.state == 0) {
        const cudaError_t e = persist_plan_build_a(h, s);
        if (e != cudaSuccess) return e;
    }
    if (h->pp_a.state != 1) return cudaErrorNotSupported;
    SolverHost& H = h->H;
    PersistDev P{};
    P.a_rp = h->A.rp;
    P.a_ci = h->A.ci;
    P.a_v = h->A.v;
    P.row_start = h->pp_a.d_row_start;
    P.win = h->pp_a.d_row_start + h->pp_a.grid + 1 + kBarWords;
    P.a_c16 = h->pp_a.d_c16;
    P.q = H.v(vXAlt);
    P.part = H.ws.partials;
    P.bar = reinterpret_cast<unsigned*>(h->pp_a.d_row_start + h->pp_a.grid + 1);
    P.err = h->d_err;
    P.sc_out = H.ws.sc;
    P.prm = H.ws.d_params;
    P.n = (int)h->A.n_rows;
    P.spin_limit = h->test_spin_limit ? h->test_spin_limit : kGridSpinLimit;
    P.silent_cta = h->test_silent_cta;
    P.b32 = H.v(vB);
    P.x32 = H.v(vX);
    const int f = h->pp_a.form;
    const void* k = f == kStreamForm   ? reinterpret_cast<const void*>(rich_persistent<kStreamForm>)
                    : f == kWindowForm ? reinterpret_cast<const void*>(rich_persistent<kWindowForm>)
                                       : reinterpret_cast<const void*>(rich_persistent<kGatherForm>);
    cudaError_t e = cudaMemsetAsync(P.bar, 0, kBarWords * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->pp_a.smem);
    if (e != cudaSuccess) return e;
    void* args[] = {&P};
    return cudaLaunchCooperativeKernel(k, dim3(h->pp_a.grid), dim3(kPNT), args, h->pp_a.smem, s);
}

void persist_plan_free(mps_csr* h) {
    dev_free(h->pp.d_row_start);
    dev_free(h->pp.d_c16);
    h->pp = PersistPlan{};
}

void persist_plan_free_all(mps_csr* h) {
    persist_plan_free(h);
    dev_free(h->pp_a.d_row_start);
    dev_free(h->pp_a.d_c16);
    h->pp_a = PersistPlan{};
}

// The reliable-update FSAI-PCG solve (x64 = FP64 solution, b64 = FP64 rhs,
// both of n entries) as one cooperative launch; the final scalars land in
// H.ws.sc like the graph form's.  Returns cudaErrorNotSupported when the
// plan says the matrix is not eligible.
cudaError_t persist_solve(mps_csr* h, const double* b64, double* x64, cudaStream_t s) {
    if (h->pp.state == 0) {
        const cudaError_t e = persist_plan_build(h, s);
        if (e != cudaSuccess) return e;
    }
    if (h->pp.state != 1) return cudaErrorNotSupported;
    SolverHost& H = h->H;
    PersistDev P{};
    P.a_rp = h->A.rp;
    P.a_ci = h->A.ci;
    P.a_v = h->A.v;
    P.m_rp = h->M.rp;
    P.m_ci = h->M.ci;
    P.m_v = h->M.v;
    P.row_start = h->pp.d_row_start;
    P.dinv = H.dinv;
    P.b = b64;
    P.x = x64;
    P.r0 = H.v(vR);
    P.r1 = H.v(vR1);
    P.p0 = H.v(vP);
    P.p1 = H.v(vP1);
    P.q = H.v(vQ);
    P.z = H.v(vW);
    P.part = H.ws.partials;
    P.bar = reinterpret_cast<unsigned*>(h->pp.d_row_start + h->pp.grid + 1);
    P.err = h->d_err;
    P.sc_out = H.ws.sc;
    P.prm = H.ws.d_params;
    P.n = (int)h->A.n_rows;
    P.spin_limit = h->test_spin_limit ? h->test_spin_limit : kGridSpinLimit;
    P.silent_cta = h->test_silent_cta;
    static_assert(4 * 3 * 1024 <= 4 * kMaxPartials, "partial slots");
    P.win = h->pp.d_row_start + h->pp.grid + 1 + kBarWords;
    P.a_c16 = h->pp.d_c16;
    P.m_c16 = h->pp.d_c16 ? h->pp.d_c16 + h->A.nnz : nullptr;
    const int f = h->pp.form;
    const void* k = f == kWindowForm   ? reinterpret_cast<const void*>(fsai_pcg_persistent<kWindowForm>)
                    : f == kStreamForm ? reinterpret_cast<const void*>(fsai_pcg_persistent<kStreamForm>)
                                       : reinterpret_cast<const void*>(fsai_pcg_persistent<kGatherForm>);
    cudaError_t e = cudaMemsetAsync(P.bar, 0, kBarWords * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->pp.smem);
    if (e != cudaSuccess) return e;
    void* args[] = {&P};
    return cudaLaunchCooperativeKernel(k, dim3(h->pp.grid), dim3(kPNT), args, h->pp.smem, s);
}

}  // namespace mps
