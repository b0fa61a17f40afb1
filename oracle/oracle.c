/*
 * oracle.c -- CPU restatement of SparseForge/mpsparse's solver path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against (tests/, __graft_entry__.smoke(), bench.py's CPU-baseline leg).  The
 * product path never links or loads it.
 *
 * Every function restates the reference algorithm from its source; the
 * reference file:line each one follows is given beside it.  Arithmetic is
 * FP64 throughout (the "FP64 host transcription"); matrix values are the FP32
 * values the caller stored.  The sort is bit-exact integer work.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* COO -> CSR                                                                */
/* ------------------------------------------------------------------------ */

static int bit_width_u32(uint32_t v) { return v ? 32 - __builtin_clz(v) : 0; }

/* iterative/BiCGSTAB/spmv.cpp:62-228.  The reference masks the 64-bit key to
 * bits(n_cols) column bits and bits(n_rows) row bits (spmv.cpp:73-77) and
 * runs one stable counting-sort pass per 4-bit digit that overlaps the mask
 * (spmv.cpp:110-170; radix_frequencies/vertical_scan/scan_histogram/reorder,
 * coo_csr.metal:17-142).  It then writes col_ind = low word, row starts where
 * the row changes, row_ptr[n] = nnz (coo_to_csr_compress, coo_csr.metal:144-178)
 * and fills empty rows backward (row_fixer, coo_csr.metal:180-193).
 * Keys outside [0,n_rows) x [0,n_cols) are undefined in the reference; here
 * they are rejected (-1).  nnz == 0 yields an all-zero row_ptr. */
int orc_coo_to_csr(const uint64_t* keys, const float* vals, uint64_t nnz,
                   uint32_t n_rows, uint32_t n_cols,
                   int32_t* row_ptr, int32_t* col_ind, float* out_vals) {
    for (uint64_t i = 0; i < nnz; ++i) {
        uint64_t r = keys[i] >> 32, c = keys[i] & 0xFFFFFFFFull;
        if (r >= n_rows || c >= n_cols) return -1;
    }
    if (nnz == 0) {
        for (uint64_t i = 0; i <= n_rows; ++i) row_ptr[i] = 0;
        return 0;
    }
    uint64_t mask = ((1ull << bit_width_u32(n_cols)) - 1) |
                    (((1ull << bit_width_u32(n_rows)) - 1) << 32);
    uint64_t* ka = (uint64_t*)malloc(nnz * sizeof(uint64_t));
    uint64_t* kb = (uint64_t*)malloc(nnz * sizeof(uint64_t));
    float* va = (float*)malloc(nnz * sizeof(float));
    float* vb = (float*)malloc(nnz * sizeof(float));
    if (!ka || !kb || !va || !vb) { free(ka); free(kb); free(va); free(vb); return -2; }
    memcpy(ka, keys, nnz * sizeof(uint64_t));
    memcpy(va, vals, nnz * sizeof(float));
    for (int shift = 0; shift < 64; shift += 4) {
        if (((0xFull << shift) & mask) == 0) continue;      /* spmv.cpp:117-122 */
        uint64_t cnt[16] = {0}, off[16];
        for (uint64_t i = 0; i < nnz; ++i) cnt[(ka[i] >> shift) & 0xF]++;
        uint64_t run = 0;
        for (int d = 0; d < 16; ++d) { off[d] = run; run += cnt[d]; }
        for (uint64_t i = 0; i < nnz; ++i) {                /* stable scatter */
            unsigned d = (unsigned)((ka[i] >> shift) & 0xF);
            kb[off[d]] = ka[i];
            vb[off[d]] = va[i];
            off[d]++;
        }
        uint64_t* tk = ka; ka = kb; kb = tk;
        float* tv = va; va = vb; vb = tv;
    }
    /* coo_to_csr_compress (coo_csr.metal:144-178) after the 0xFF fill
     * (spmv.cpp:187-191). */
    for (uint64_t i = 0; i <= n_rows; ++i) row_ptr[i] = (int32_t)0xFFFFFFFF;
    for (uint64_t g = 0; g < nnz; ++g) {
        uint32_t row = (uint32_t)(ka[g] >> 32);
        col_ind[g] = (int32_t)(uint32_t)(ka[g] & 0xFFFFFFFFull);
        if (g == 0) {
            row_ptr[0] = 0;
            row_ptr[row] = 0;
        } else if (row != (uint32_t)(ka[g - 1] >> 32)) {
            row_ptr[row] = (int32_t)g;
        }
        if (g == nnz - 1) row_ptr[n_rows] = (int32_t)nnz;
    }
    /* row_fixer (coo_csr.metal:180-193). */
    for (int64_t i = (int64_t)n_rows - 1; i >= 0; --i)
        if ((uint32_t)row_ptr[i] == 0xFFFFFFFFu) row_ptr[i] = row_ptr[i + 1];
    memcpy(out_vals, va, nnz * sizeof(float));
    free(ka); free(kb); free(va); free(vb);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* SpMV                                                                      */
/* ------------------------------------------------------------------------ */

/* spmv_op, iterative/BiCGSTAB/spmv.metal:11-49: one row, sum of val*x[col]. */
void orc_csr_spmv(const int32_t* rp, const int32_t* ci, const float* v,
                  int64_t n, const double* x, double* y, int threads) {
    (void)threads;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : 1)
#endif
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) s += (double)v[k] * x[ci[k]];
        y[i] = s;
    }
}

/* spmv_op, iterative/BiCGSTAB/bcsr_spmv.metal:30-69: block row br produces
 * y[B*br + k] = sum over blocks of dot(block row k, x[B*bc .. B*bc+B-1]);
 * blocks are row-major B x B (scipy bsr.data.flatten(), bcsr_benchmark.py:52). */
void orc_bcsr_spmv(const int32_t* rp, const int32_t* ci, const float* v,
                   int64_t nbr, int B, const double* x, double* y) {
    for (int64_t br = 0; br < nbr; ++br) {
        for (int k = 0; k < B; ++k) y[br * B + k] = 0.0;
        for (int32_t j = rp[br]; j < rp[br + 1]; ++j) {
            const float* blk = v + (int64_t)j * B * B;
            const double* xs = x + (int64_t)ci[j] * B;
            for (int k = 0; k < B; ++k) {
                double s = 0.0;
                for (int c = 0; c < B; ++c) s += (double)blk[k * B + c] * xs[c];
                y[br * B + k] += s;
            }
        }
    }
}

static void apply(const orc_op* A, const double* x, double* y, int threads) {
    if (A->block == 0)
        orc_csr_spmv(A->row_ptr, A->col_ind, A->val, A->n, x, y, threads);
    else
        orc_bcsr_spmv(A->row_ptr, A->col_ind, A->val, A->n / A->block, A->block, x, y);
}

/* Deterministic dot: fixed static chunks summed in chunk order. */
static double dot(const double* a, const double* b, int64_t n, int threads) {
    int t = threads > 0 ? threads : 1;
    if (t == 1) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
        return s;
    }
    double part[256] = {0};
    if (t > 256) t = 256;
    int64_t chunk = (n + t - 1) / t;
#ifdef _OPENMP
#pragma omp parallel for schedule(static, 1) num_threads(t)
#endif
    for (int c = 0; c < t; ++c) {
        int64_t lo = (int64_t)c * chunk, hi = lo + chunk < n ? lo + chunk : n;
        double s = 0.0;
        for (int64_t i = lo; i < hi; ++i) s += a[i] * b[i];
        part[c] = s;
    }
    double s = 0.0;
    for (int c = 0; c < t; ++c) s += part[c];
    return s;
}

/* Row chunk c of t (the chunks dot() sums in order). */
static void chunk_of(int64_t n, int t, int c, int64_t* lo, int64_t* hi) {
    int64_t chunk = (n + t - 1) / t;
    *lo = (int64_t)c * chunk;
    *hi = *lo + chunk < n ? *lo + chunk : n;
    if (*lo > n) *lo = n;
}

/* q = A p (CSR) and p.q with the chunking and order of dot(): the same
 * numbers as orc_csr_spmv followed by dot(p, q), in one parallel pass. */
static double spmv_dot(const orc_op* A, const double* p, double* q, int threads) {
    int t = threads > 0 ? threads : 1;
    if (t > 256) t = 256;
    double part[256] = {0};
#ifdef _OPENMP
#pragma omp parallel for schedule(static, 1) num_threads(t)
#endif
    for (int c = 0; c < t; ++c) {
        int64_t lo, hi;
        chunk_of(A->n, t, c, &lo, &hi);
        double s = 0.0;
        for (int64_t i = lo; i < hi; ++i) {
            double y = 0.0;
            for (int32_t k = A->row_ptr[i]; k < A->row_ptr[i + 1]; ++k)
                y += (double)A->val[k] * p[A->col_ind[k]];
            q[i] = y;
            s += p[i] * y;
        }
        part[c] = s;
    }
    double s = 0.0;
    for (int c = 0; c < t; ++c) s += part[c];
    return s;
}

/* x += alpha p, r -= alpha q, then r.r and (Jacobi) z = D^-1 r, r.z, in one
 * parallel pass with dot()'s chunking and order. */
static void update_xr(double* x, double* r, double* z, const double* p, const double* q,
                      const double* dinv, double alpha, int64_t n, int threads, double* rr,
                      double* rz) {
    int t = threads > 0 ? threads : 1;
    if (t > 256) t = 256;
    double prr[256] = {0}, prz[256] = {0};
#ifdef _OPENMP
#pragma omp parallel for schedule(static, 1) num_threads(t)
#endif
    for (int c = 0; c < t; ++c) {
        int64_t lo, hi;
        chunk_of(n, t, c, &lo, &hi);
        double s = 0.0, sz = 0.0;
        for (int64_t k = lo; k < hi; ++k) {
            x[k] += alpha * p[k];
            r[k] -= alpha * q[k];
            s += r[k] * r[k];
            if (dinv) {
                z[k] = dinv[k] * r[k];
                sz += r[k] * z[k];
            }
        }
        prr[c] = s;
        prz[c] = sz;
    }
    double s = 0.0, sz = 0.0;
    for (int c = 0; c < t; ++c) {
        s += prr[c];
        sz += prz[c];
    }
    *rr = s;
    *rz = dinv ? sz : s;
}

/* p = zz + beta p */
static void axpby_p(double* p, const double* zz, double beta, int64_t n, int threads) {
    int t = threads > 0 ? threads : 1;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(t)
#endif
    for (int64_t k = 0; k < n; ++k) p[k] = zz[k] + beta * p[k];
}

static void diag_of(const orc_op* A, double* d) {
    for (int64_t i = 0; i < A->n; ++i) d[i] = 0.0;
    if (A->block == 0) {
        for (int64_t i = 0; i < A->n; ++i)
            for (int32_t k = A->row_ptr[i]; k < A->row_ptr[i + 1]; ++k)
                if (A->col_ind[k] == i) d[i] += A->val[k];
    } else {
        int B = A->block;
        for (int64_t br = 0; br < A->n / B; ++br)
            for (int32_t j = A->row_ptr[br]; j < A->row_ptr[br + 1]; ++j)
                if (A->col_ind[j] == br)
                    for (int k = 0; k < B; ++k) d[br * B + k] += A->val[(int64_t)j * B * B + k * B + k];
    }
}

double orc_true_residual(const orc_op* A, const double* b, const double* x) {
    double* ax = (double*)malloc(A->n * sizeof(double));
    apply(A, x, ax, 1);
    double rr = 0.0, bb = 0.0;
    for (int64_t i = 0; i < A->n; ++i) {
        double r = b[i] - ax[i];
        rr += r * r;
        bb += b[i] * b[i];
    }
    free(ax);
    return bb > 0 ? sqrt(rr / bb) : sqrt(rr);
}

/* ------------------------------------------------------------------------ */
/* CG                                                                        */
/* ------------------------------------------------------------------------ */

/* csr_tensor::cgd_op, iterative/BiCGSTAB/spmv.cpp:528-659, kernels
 * update_xr / update_p (cgd.metal:11-82):
 *   x = 0, r = p = b, rr = r.r                       (spmv.cpp:542-565)
 *   loop i < min(1000, n)                             (spmv.cpp:572-573)
 *     Ap = A p, pAp = p.Ap                            (fused_spvmv)
 *     alpha = |pAp| > 1e-9 ? rr/pAp : 0               (cgd.metal:38-42)
 *     x += alpha p, r -= alpha Ap, rr' = r.r          (cgd.metal:44-46)
 *     p = r + (rr'/rr) p                              (cgd.metal:81)
 *     every 50 iterations stop if rr (the value before this update) < 1e-5
 *     (spmv.cpp:603-627; the curr/next swap happens after the check).
 * compat = 0: x0 = 0, relative test ||r|| <= tol ||b|| after every update,
 * optional Jacobi preconditioner (z = r / diag(A)). */
int orc_cg(const orc_op* A, const double* b, double* x, const orc_opts* o, orc_info* info) {
    int64_t n = A->n;
    int th = o->threads;
    double *r = malloc(n * 8), *p = malloc(n * 8), *q = malloc(n * 8), *z = malloc(n * 8),
           *dinv = NULL;
    if (o->precond == 1 && !o->compat) {
        dinv = malloc(n * 8);
        diag_of(A, dinv);
        for (int64_t i = 0; i < n; ++i) dinv[i] = dinv[i] != 0.0 ? 1.0 / dinv[i] : 1.0;
    }
    for (int64_t i = 0; i < n; ++i) {
        x[i] = 0.0;
        r[i] = b[i];
        z[i] = dinv ? dinv[i] * b[i] : b[i];
        p[i] = z[i];
    }
    double bnorm = sqrt(dot(b, b, n, th));
    double rr = dot(r, r, n, th);
    double rz = dinv ? dot(r, z, n, th) : rr;
    int cap = o->compat ? (n < 1000 ? (int)n : 1000) : o->max_iter;
    info->iters = 0;
    info->converged = 0;
    info->breakdown = 0;
    if (!o->compat && bnorm == 0.0) {
        info->converged = 1;
        info->rel_resid = 0.0;
        goto done;
    }
    for (int i = 0; i < cap; ++i) {
        double pq;
        if (A->block == 0) {
            pq = spmv_dot(A, p, q, th);               /* q = A p and p.q, one pass */
        } else {
            apply(A, p, q, th);
            pq = dot(p, q, n, th);
        }
        double alpha;
        if (o->compat) {
            alpha = fabs(pq) > 1e-9 ? rz / pq : 0.0;
        } else {
            if (!(pq > 0.0)) { info->breakdown = 1; break; }
            alpha = rz / pq;
        }
        double rr_new, rz_new;
        update_xr(x, r, z, p, q, dinv, alpha, n, th, &rr_new, &rz_new);
        double beta = rz_new / rz;
        const double* zz = dinv ? z : r;
        axpby_p(p, zz, beta, n, th);
        info->iters = i + 1;
        if (o->compat) {
            if (i % 50 == 0 && rr < 1e-5) { rr = rr_new; info->converged = 1; break; }
        } else if (sqrt(rr_new) <= o->tol * bnorm) {
            rr = rr_new;
            info->converged = 1;
            break;
        }
        rr = rr_new;
        rz = rz_new;
    }
    info->rel_resid = bnorm > 0 ? sqrt(rr) / bnorm : sqrt(rr);
done:
    free(r); free(p); free(q); free(z); free(dinv);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* BiCGSTAB                                                                  */
/* ------------------------------------------------------------------------ */

/* csr_tensor::bicgstab_op, iterative/BiCGSTAB/spmv.cpp:699-888, kernels upp,
 * fused_spvmv, f_upalpha_ups, spmv_op, f_dip, f_upomega_upxr_laa
 * (bicgstab.metal:12-326).  Scalar slots {rho_prev, rho_curr, alpha, omega,
 * sigma, phi1, phi2, ||r||^2} start at {1,1,1,1,0,0,0,0} (spmv.cpp:724) and
 * the first r.r is added on top of slot 1 (spmv.cpp:744-752), so compat mode
 * starts from rho0 = 1 + b.b.  Guards: beta = 0 unless |rho_old| > 1e-15 and
 * |omega| > 1e-15, and beta = 0 if it is inf/NaN (bicgstab.metal:46-56);
 * omega = 0 if |phi2| < 1e-20 (bicgstab.metal:264-269).  The compat stop rule
 * models the reference's delayed check (spmv.cpp:835-859) without its host
 * race: the first check index j (a multiple of 50, j + 50 < cap) whose
 * ||r_j||^2 < 1e-5 returns the iterate after iteration j; the cap is
 * min(5000, n).  compat = 0 is the plain van der Vorst recurrence with
 * rho0 = b.b and the relative test every iteration. */
int orc_bicgstab(const orc_op* A, const double* b, double* x, const orc_opts* o, orc_info* info) {
    int64_t n = A->n;
    int th = o->threads;
    double *r = malloc(n * 8), *r0 = malloc(n * 8), *p = malloc(n * 8), *v = malloc(n * 8),
           *s = malloc(n * 8), *t = malloc(n * 8), *xs = NULL;
    for (int64_t i = 0; i < n; ++i) {
        x[i] = 0.0;
        r[i] = r0[i] = p[i] = b[i];
        v[i] = 0.0;
    }
    double bnorm = sqrt(dot(b, b, n, th));
    double rho_old = 1.0, alpha = 1.0, omega = 1.0;
    double rho = (o->compat ? 1.0 : 0.0) + dot(r, r, n, th);
    double rnorm2 = rho - (o->compat ? 1.0 : 0.0);
    int cap = o->compat ? (n < 5000 ? (int)n : 5000) : o->max_iter;
    double staged = 1e9;          /* host copy of ||r||^2 from the last check */
    if (o->compat) xs = malloc(n * 8);
    info->iters = 0;
    info->converged = 0;
    info->breakdown = 0;
    if (!o->compat && bnorm == 0.0) {
        info->converged = 1;
        info->rel_resid = 0.0;
        goto done;
    }
    for (int i = 0; i < cap; ++i) {
        if (i > 0) {                                          /* upp */
            double beta = 0.0;
            if (fabs(rho_old) > 1e-15 && fabs(omega) > 1e-15) {
                beta = (rho / rho_old) * (alpha / omega);
                if (isinf(beta) || isnan(beta)) beta = 0.0;
            }
            for (int64_t k = 0; k < n; ++k) p[k] = r[k] + beta * (p[k] - omega * v[k]);
        } else {
            for (int64_t k = 0; k < n; ++k) p[k] = r[k];
        }
        apply(A, p, v, th);                                   /* fused_spvmv */
        double sigma = dot(r0, v, n, th);
        if (!o->compat && sigma == 0.0) { info->breakdown = 1; break; }
        alpha = rho / sigma;                                  /* f_upalpha_ups */
        for (int64_t k = 0; k < n; ++k) s[k] = r[k] - alpha * v[k];
        apply(A, s, t, th);                                   /* spmv_op */
        double phi1 = dot(t, s, n, th), phi2 = dot(t, t, n, th);   /* f_dip */
        omega = fabs(phi2) < 1e-20 ? 0.0 : phi1 / phi2;       /* f_upomega_upxr_laa */
        for (int64_t k = 0; k < n; ++k) {
            x[k] += alpha * p[k] + omega * s[k];
            r[k] = s[k] - omega * t[k];
        }
        rho_old = rho;
        rho = dot(r0, r, n, th);
        rnorm2 = dot(r, r, n, th);
        info->iters = i + 1;
        if (o->compat) {
            if (i % 50 == 0) {
                if (i > 0 && staged < 1e-5) {
                    /* the batch after the previous check is discarded */
                    memcpy(x, xs, n * 8);
                    info->iters = i - 50 + 1;
                    info->converged = 1;
                    rnorm2 = staged;
                    break;
                }
                staged = rnorm2;
                memcpy(xs, x, n * 8);
            }
        } else {
            if (sqrt(rnorm2) <= o->tol * bnorm) { info->converged = 1; break; }
            if (omega == 0.0 || rho == 0.0) { info->breakdown = 1; break; }
        }
    }
    info->rel_resid = bnorm > 0 ? sqrt(rnorm2) / bnorm : sqrt(rnorm2);
done:
    free(r); free(r0); free(p); free(v); free(s); free(t); free(xs);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Richardson                                                                */
/* ------------------------------------------------------------------------ */

/* csr_tensor::iterative_op / iterative_step, iterative/richardson/spmv.cpp:
 * 376-425 and 441-495: x = 0, then for a fixed count s1 = A x,
 * s2 = w b + (-w) s1, x = x + s2 (weighted_add, richardson/spmv.metal:50-63).
 * compat = 1 fixes w = 0.01 and 1000 iterations (spmv.cpp:402-404). */
int orc_richardson(const orc_op* A, const double* b, double* x, const orc_opts* o, orc_info* info) {
    int64_t n = A->n;
    double w = o->compat ? 0.01 : o->omega;
    int iters = o->compat ? 1000 : o->max_iter;
    double* s1 = malloc(n * 8);
    for (int64_t i = 0; i < n; ++i) x[i] = 0.0;
    for (int it = 0; it < iters; ++it) {
        apply(A, x, s1, o->threads);
        for (int64_t i = 0; i < n; ++i) x[i] = x[i] + (w * b[i] + (-w) * s1[i]);
    }
    info->iters = iters;
    info->converged = 0;
    info->breakdown = 0;
    info->rel_resid = orc_true_residual(A, b, x);
    free(s1);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Learned FSAI (no reference counterpart: restates this package's design)  */
/* ------------------------------------------------------------------------ */

int64_t orc_fsai_pattern(const orc_op* A, int32_t* g_rp, int32_t* g_ci, int32_t* g_row,
                         int32_t* g_aidx) {
    int64_t k = 0;
    g_rp[0] = 0;
    for (int64_t i = 0; i < A->n; ++i) {
        for (int32_t a = A->row_ptr[i]; a < A->row_ptr[i + 1]; ++a) {
            if (A->col_ind[a] <= i) {
                g_ci[k] = A->col_ind[a];
                g_row[k] = (int32_t)i;
                g_aidx[k] = a;
                ++k;
            }
        }
        g_rp[i + 1] = (int32_t)k;
    }
    return k;
}

typedef struct {
    double diag, dd;
    int32_t ln, lf, un, uf;     /* nearest / farther lower and upper neighbours (-1: none) */
    double lnv, lfv, unv, ufv;  /* their coefficients */
} orc_rowinfo;

static void row_info(const orc_op* A, int64_t i, orc_rowinfo* ri) {
    ri->diag = 0.0;
    ri->ln = ri->lf = ri->un = ri->uf = -1;
    ri->lnv = ri->lfv = ri->unv = ri->ufv = 0.0;
    double off = 0.0;
    for (int32_t a = A->row_ptr[i]; a < A->row_ptr[i + 1]; ++a) {
        const int32_t c = A->col_ind[a];
        const double v = A->val[a];
        if (c == i) {
            ri->diag += v;
            continue;
        }
        off += fabs(v);
        if (c < i) {          /* columns ascend: the last lower ones are nearest */
            ri->lf = ri->ln;
            ri->lfv = ri->lnv;
            ri->ln = c;
            ri->lnv = v;
        } else if (ri->un < 0) {
            ri->un = c;
            ri->unv = v;
        } else if (ri->uf < 0) {
            ri->uf = c;
            ri->ufv = v;
        }
    }
    ri->dd = ri->diag != 0.0 ? (ri->diag - off) / ri->diag : 0.0;
}

static double diag_at(const orc_op* A, int64_t i) {
    double d = 0.0;
    for (int32_t a = A->row_ptr[i]; a < A->row_ptr[i + 1]; ++a)
        if (A->col_ind[a] == i) d += A->val[a];
    return d;
}

static double nrm(double v, double di, double dj) { return v / sqrt(di * dj); }

void orc_fsai_features(const orc_op* A, int64_t nnz_g, const int32_t* g_row, const int32_t* g_ci,
                       const int32_t* g_aidx, float* X) {
    for (int64_t k = 0; k < nnz_g; ++k) {
        const int64_t i = g_row[k], j = g_ci[k];
        orc_rowinfo ri, rj;
        row_info(A, i, &ri);
        row_info(A, j, &rj);
        const double di = ri.diag, dj = rj.diag;
        float* f = X + k * ORC_NF;
        f[0] = 1.0f;
        f[1] = (float)(i == j);
        f[2] = (float)(j == ri.ln);
        f[3] = (float)(j == ri.lf);
        f[4] = ri.ln >= 0 ? (float)nrm(ri.lnv, di, diag_at(A, ri.ln)) : 0.0f;
        f[5] = ri.lf >= 0 ? (float)nrm(ri.lfv, di, diag_at(A, ri.lf)) : 0.0f;
        f[6] = ri.un >= 0 ? (float)nrm(ri.unv, di, diag_at(A, ri.un)) : 0.0f;
        f[7] = ri.uf >= 0 ? (float)nrm(ri.ufv, di, diag_at(A, ri.uf)) : 0.0f;
        f[8] = ri.ln >= 0 ? (float)log(di / diag_at(A, ri.ln)) : 0.0f;
        f[9] = ri.lf >= 0 ? (float)log(di / diag_at(A, ri.lf)) : 0.0f;
        f[10] = i == j ? 1.0f : (float)nrm(A->val[g_aidx[k]], di, dj);
        f[11] = (float)log(di / dj);
        f[12] = (float)ri.dd;
        f[13] = (float)rj.dd;
        f[14] = rj.ln >= 0 ? (float)nrm(rj.lnv, dj, diag_at(A, rj.ln)) : 0.0f;
        f[15] = rj.lf >= 0 ? (float)nrm(rj.lfv, dj, diag_at(A, rj.lf)) : 0.0f;
    }
}

/* Round-to-nearest-even to bfloat16 (kept as a float). */
static float bf16r(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return f;       /* inf / nan */
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

/* The network's activation: GELU in its tanh form (Hendrycks & Gimpel 2016),
 * 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))), and its derivative. */
static double gelu(double x) {
    const double c = sqrt(2.0 / M_PI);
    return 0.5 * x * (1.0 + tanh(c * (x + 0.044715 * x * x * x)));
}
static double gelu_d(double x) {
    const double c = sqrt(2.0 / M_PI);
    const double t = tanh(c * (x + 0.044715 * x * x * x));
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * c * (1.0 + 3.0 * 0.044715 * x * x);
}

typedef struct {
    const float *W1, *b1, *W2, *b2, *w3, *b3;
} orc_mlp;

static orc_mlp mlp_view(const float* p) {
    orc_mlp m;
    m.W1 = p;
    m.b1 = m.W1 + ORC_NF * ORC_NH;
    m.W2 = m.b1 + ORC_NH;
    m.b2 = m.W2 + ORC_NH * ORC_NH;
    m.w3 = m.b2 + ORC_NH;
    m.b3 = m.w3 + ORC_NH;
    return m;
}

/* One row through the network; z1, h1 (bf16-rounded), z2, h2 out. */
static double mlp_row(const orc_mlp* m, const float* x, double* z1, double* h1, double* z2,
                      double* h2) {
    float xb[ORC_NF];
    for (int f = 0; f < ORC_NF; ++f) xb[f] = bf16r(x[f]);
    for (int o = 0; o < ORC_NH; ++o) {
        double s = 0.0;
        for (int f = 0; f < ORC_NF; ++f) s += (double)xb[f] * bf16r(m->W1[f * ORC_NH + o]);
        z1[o] = s + m->b1[o];
        h1[o] = bf16r((float)gelu(z1[o]));
    }
    double out = m->b3[0];
    for (int o = 0; o < ORC_NH; ++o) {
        double s = 0.0;
        for (int f = 0; f < ORC_NH; ++f) s += h1[f] * bf16r(m->W2[f * ORC_NH + o]);
        z2[o] = s + m->b2[o];
        h2[o] = gelu(z2[o]);
        out += h2[o] * bf16r(m->w3[o]);
    }
    return out;
}

void orc_mlp_forward(const float* params, const float* X, int64_t N, double* out) {
    orc_mlp m = mlp_view(params);
    double z1[ORC_NH], h1[ORC_NH], z2[ORC_NH], h2[ORC_NH];
    for (int64_t r = 0; r < N; ++r) out[r] = mlp_row(&m, X + r * ORC_NF, z1, h1, z2, h2);
}

void orc_mlp_backward(const float* params, const float* X, int64_t N, const double* dout,
                      double* grad) {
    orc_mlp m = mlp_view(params);
    for (int i = 0; i < ORC_NPARAM; ++i) grad[i] = 0.0;
    double *gW1 = grad, *gb1 = gW1 + ORC_NF * ORC_NH, *gW2 = gb1 + ORC_NH,
           *gb2 = gW2 + ORC_NH * ORC_NH, *gw3 = gb2 + ORC_NH, *gb3 = gw3 + ORC_NH;
    double z1[ORC_NH], h1[ORC_NH], z2[ORC_NH], h2[ORC_NH], dz2[ORC_NH], dz1[ORC_NH];
    for (int64_t r = 0; r < N; ++r) {
        const float* x = X + r * ORC_NF;
        mlp_row(&m, x, z1, h1, z2, h2);
        const double d = dout[r];
        gb3[0] += d;
        for (int o = 0; o < ORC_NH; ++o) {
            gw3[o] += d * h2[o];
            const double g = d * bf16r(m.w3[o]) * gelu_d(z2[o]);
            gb2[o] += g;
            dz2[o] = bf16r((float)g);
        }
        for (int f = 0; f < ORC_NH; ++f)
            for (int o = 0; o < ORC_NH; ++o) gW2[f * ORC_NH + o] += h1[f] * dz2[o];
        for (int f = 0; f < ORC_NH; ++f) {
            double s = 0.0;
            for (int o = 0; o < ORC_NH; ++o) s += dz2[o] * bf16r(m.W2[f * ORC_NH + o]);
            const double g = s * gelu_d(z1[f]);
            gb1[f] += g;
            dz1[f] = bf16r((float)g);
        }
        for (int f = 0; f < ORC_NF; ++f) {
            const double xb = bf16r(x[f]);
            for (int o = 0; o < ORC_NH; ++o) gW1[f * ORC_NH + o] += xb * dz1[o];
        }
    }
}

static void apply_t(const orc_op* G, const double* v, double* u) {   /* u = G^T v */
    for (int64_t j = 0; j < G->n; ++j) u[j] = 0.0;
    for (int64_t i = 0; i < G->n; ++i)
        for (int32_t a = G->row_ptr[i]; a < G->row_ptr[i + 1]; ++a)
            u[G->col_ind[a]] += (double)G->val[a] * v[i];
}

double orc_fsai_probe_loss_grad(const orc_op* A, const orc_op* G, const double* V, int k,
                                double* grad_g) {
    const int64_t n = A->n;
    double *u = malloc(n * 8), *w = malloc(n * 8), *y = malloc(n * 8), *e = malloc(n * 8),
           *t = malloc(n * 8), *s = malloc(n * 8);
    const int64_t nnz = G->row_ptr[n];
    for (int64_t a = 0; a < nnz; ++a) grad_g[a] = 0.0;
    double loss = 0.0;
    for (int p = 0; p < k; ++p) {
        const double* v = V + (int64_t)p * n;
        apply_t(G, v, u);
        apply(A, u, w, 1);
        apply(G, w, y, 1);
        for (int64_t i = 0; i < n; ++i) {
            e[i] = y[i] - v[i];
            loss += e[i] * e[i];
        }
        apply_t(G, e, t);
        apply(A, t, s, 1);
        for (int64_t i = 0; i < n; ++i)
            for (int32_t a = G->row_ptr[i]; a < G->row_ptr[i + 1]; ++a) {
                const int32_t j = G->col_ind[a];
                grad_g[a] += e[i] * w[j] + v[i] * s[j];
            }
    }
    const double sc = 1.0 / ((double)k * (double)n);
    for (int64_t a = 0; a < nnz; ++a) grad_g[a] *= 2.0 * sc;
    free(u); free(w); free(y); free(e); free(t); free(s);
    return loss * sc;
}
