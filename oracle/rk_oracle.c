/*
 * CPU oracle for the relativistic R^k / Y^k path — TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the reference algorithm that the B200 engine
 * must reproduce.  It is used by the test-suite as the checker, by the smoke
 * entry as the checker, and by the benchmark's CPU-baseline leg as the timed
 * reference-algorithm port.  Nothing in the shipped engine links or calls it.
 *
 * Restated functions (atomx, path relative to its project root):
 *   oracle_yk_row     <- src/atomx/numerics/yk.py:88-154  (yk_flat)
 *       outward cell sums with the interpolatory partial matrix `mo`, inward
 *       cell sums with `mi`, then Y_i = r_i^-(k+1) I_out + r_i^k I_in.
 *       The loop order and the left-to-right product order
 *       ((w*rho)*r^k)*mo are the same as the reference, so results agree
 *       to the last bit when r^k agrees.
 *   oracle_int_pow    <- Numba's float**int lowering used by yk.py:116-117
 *       (square-and-multiply; negative powers as 1/x^|n|).
 *   oracle_dot_table  <- src/atomx/numerics/bspline/slater.py:118-130
 *       (slater_rk_poisson: R = sum_i w_i rho13_i Y[rho24]_i), one plain
 *       dot per ordered table entry, as the reference evaluates it per
 *       integral; oracle_dot_block is the same dot over a block of a table.
 *
 *   oracle_grid_*     <- src/atomx/numerics/quadrature.py:247-391 (trapezoid Y^k
 *       on arbitrary grids; see the section at the end of this file).
 *
 * Parity of this oracle is pinned by tests against golden vectors produced by
 * running the reference itself (tests/golden/make_golden.py).
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* Minimal static-partition parallel-for over [0, count) with POSIX threads. */
typedef void (*range_fn)(void *ctx, long lo, long hi);
struct range_job { range_fn fn; void *ctx; long lo, hi; };

static void *range_thread(void *arg)
{
    struct range_job *j = (struct range_job *)arg;
    j->fn(j->ctx, j->lo, j->hi);
    return NULL;
}

int oracle_max_threads(void)
{
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

static void parallel_for(range_fn fn, void *ctx, long count, int threads)
{
    if (threads <= 0) threads = oracle_max_threads();
    if (threads > 256) threads = 256;
    if ((long)threads > count) threads = count > 0 ? (int)count : 1;
    if (threads <= 1) { fn(ctx, 0, count); return; }
    pthread_t tid[256];
    struct range_job jobs[256];
    int started = 0;
    for (int t = 0; t < threads; ++t) {
        jobs[t].fn = fn; jobs[t].ctx = ctx;
        jobs[t].lo = count * t / threads; jobs[t].hi = count * (t + 1) / threads;
        if (pthread_create(&tid[t], NULL, range_thread, &jobs[t]) == 0) ++started;
        else { fn(ctx, jobs[t].lo, jobs[t].hi); tid[t] = 0; }
    }
    for (int t = 0; t < threads; ++t)
        if (tid[t]) pthread_join(tid[t], NULL);
    (void)started;
}

double oracle_int_pow(double x, long n)
{
    int invert = n < 0;
    unsigned long e = invert ? (unsigned long)(-n) : (unsigned long)n;
    double r = 1.0, a = x;
    while (e != 0) {
        if (e & 1UL) r *= a;
        e >>= 1;
        a *= a;
    }
    return invert ? 1.0 / r : r;
}

/* One Y^k row.  rho, r, w, yk have n = nv*ng entries; mo, mi are ng*ng,
 * row-major.  scratch must hold 4*n doubles. */
void oracle_yk_row(const double *rho, const double *r, const double *w,
                   long n, int k, int nv, int ng,
                   const double *mo, const double *mi,
                   double *yk, double *scratch)
{
    double *rk = scratch, *rkm = scratch + n, *iout = scratch + 2 * n, *iin = scratch + 3 * n;
    for (long i = 0; i < n; ++i) {
        rk[i] = oracle_int_pow(r[i], k);
        rkm[i] = oracle_int_pow(r[i], -(long)(k + 1));
    }
    double base = 0.0;
    for (int m = 0; m < nv; ++m) {
        long off = (long)m * ng;
        for (int i = 0; i < ng; ++i) {
            double s = base;
            for (int j = 0; j < ng; ++j)
                s += w[off + j] * rho[off + j] * rk[off + j] * mo[i * ng + j];
            iout[off + i] = s;
        }
        for (int j = 0; j < ng; ++j)
            base += w[off + j] * rho[off + j] * rk[off + j];
    }
    base = 0.0;
    for (int m = nv - 1; m >= 0; --m) {
        long off = (long)m * ng;
        for (int i = 0; i < ng; ++i) {
            double s = base;
            for (int j = 0; j < ng; ++j)
                s += w[off + j] * rho[off + j] * rkm[off + j] * mi[i * ng + j];
            iin[off + i] = s;
        }
        for (int j = 0; j < ng; ++j)
            base += w[off + j] * rho[off + j] * rkm[off + j];
    }
    for (long i = 0; i < n; ++i)
        yk[i] = rkm[i] * iout[i] + rk[i] * iin[i];
}

struct yk_rows_ctx {
    const double *rho, *r, *w, *mo, *mi; const int *ks; double *yk; int nv, ng;
};

static void yk_rows_range(void *vctx, long lo, long hi)
{
    struct yk_rows_ctx *c = (struct yk_rows_ctx *)vctx;
    long n = (long)c->nv * c->ng;
    double *scratch = (double *)malloc(sizeof(double) * 4 * (size_t)n);
    if (!scratch) return;
    for (long q = lo; q < hi; ++q)
        oracle_yk_row(c->rho + q * n, c->r, c->w, n, c->ks[q], c->nv, c->ng,
                      c->mo, c->mi, c->yk + q * n, scratch);
    free(scratch);
}

/* Many rows: row q uses density rho[q*n..] and multipole ks[q]. */
void oracle_yk_rows(const double *rho, const int *ks, long nrows,
                    const double *r, const double *w, int nv, int ng,
                    const double *mo, const double *mi, double *yk, int threads)
{
    struct yk_rows_ctx c = {rho, r, w, mo, mi, ks, yk, nv, ng};
    parallel_for(yk_rows_range, &c, nrows, threads);
}

/* R[e] = sum_i g[ia[e]][i] * y[ib[e]][i] for each listed entry e, with
 * g = w*rho13 rows and y = Y^k rows, both of length n.  One dot per entry. */
struct dot_ctx { const double *g, *y; const long *ia, *ib; double *out; long n; };

static void dot_range(void *vctx, long lo, long hi)
{
    struct dot_ctx *c = (struct dot_ctx *)vctx;
    for (long e = lo; e < hi; ++e) {
        const double *a = c->g + c->ia[e] * c->n, *b = c->y + c->ib[e] * c->n;
        double s = 0.0;
        for (long i = 0; i < c->n; ++i) s += a[i] * b[i];
        c->out[e] = s;
    }
}

void oracle_dot_table(const double *g, const double *y, long n,
                      const long *ia, const long *ib, long nent,
                      double *out, int threads)
{
    struct dot_ctx c = {g, y, ia, ib, out, n};
    parallel_for(dot_range, &c, nent, threads);
}

/* out[j*na + i] = sum_x g[i][x] * y[j][x] for every i < na, j < nb: the
 * per-entry dot of oracle_dot_table over a block of a table (every row a of a
 * multipole group against the Y^k rows b listed in y), without index arrays.
 * One plain dot per ordered entry, as slater.py:130 evaluates each integral. */
struct block_ctx { const double *g, *y; double *out; long n, na; };

static void block_range(void *vctx, long lo, long hi)
{
    struct block_ctx *c = (struct block_ctx *)vctx;
    for (long j = lo; j < hi; ++j) {
        const double *b = c->y + j * c->n;
        double *o = c->out + j * c->na;
        for (long i = 0; i < c->na; ++i) {
            const double *a = c->g + i * c->n;
            double s = 0.0;
            for (long x = 0; x < c->n; ++x) s += a[x] * b[x];
            o[i] = s;
        }
    }
}

void oracle_dot_block(const double *g, long na, const double *y, long nb, long n, double *out, int threads)
{
    struct block_ctx c = {g, y, out, n, na};
    parallel_for(block_range, &c, nb, threads);
}

/* ------------------------------------------------------------------------
 * Arbitrary-grid trapezoid Y^k (atomx src/atomx/numerics/quadrature.py).
 *
 * oracle_grid_yk_rho    <- quadrature.py:247-279 (_yk_kernel_rho)
 * oracle_grid_pair_yk   <- quadrature.py:313-352 (_pair_yk: fused density)
 * oracle_grid_slater_rk <- quadrature.py:375-391 (_slater_rk_kernel)
 * oracle_grid_pair_dot_batch <- quadrature.py:282-310, 355-372
 *
 * The tables rk / inverse (block-scaled powers), the block starts `cuts`
 * and the frame transfers come from the numpy restatement of
 * _coulomb_tables (quadrature.py:190-231) in oracle.py.  The scans run in the
 * reference's order: inward cumulative trapezoids from the last node, the
 * carry rescaled by the transfer at each block change, then outward with
 * y_i = inner_i * inverse_i + rk_i * y_i.  Each expression keeps the
 * reference's operation order.  Pinned results: bit-identical for the batch
 * and Y^k functions; for grid_slater_rk with nonzero small components the
 * reference (one Numba function with the scan inlined) rounds a few
 * multiply-adds as fused operations, and the values agree to ~1e-16.
 * ------------------------------------------------------------------------ */
#define GRID_SCAN(DENS)                                                        \
    do {                                                                       \
        double acc = 0.0, prev = (DENS(n - 1)) * inverse[n - 1];               \
        if (i_cut == n - 1) y[n - 1] = 0.0;                                    \
        for (long block = ncuts - 2; block >= 0; --block) {                    \
            if (block < ncuts - 2) {                                           \
                acc *= transfer[block];                                        \
                prev *= transfer[block];                                       \
            }                                                                  \
            long top = cuts[block + 1] - 1 < n - 2 ? cuts[block + 1] - 1 : n - 2; \
            for (long i = top; i >= cuts[block]; --i) {                        \
                double b = (DENS(i)) * inverse[i];                             \
                acc += .5 * (b + prev) * (r[i + 1] - r[i]);                    \
                if (i <= i_cut) y[i] = acc;                                    \
                prev = b;                                                      \
            }                                                                  \
        }                                                                      \
        double inner = 0.0;                                                    \
        prev = (DENS(0)) * rk[0];                                              \
        y[0] *= rk[0];                                                         \
        for (long block = 0; block < ncuts - 1; ++block) {                     \
            if (cuts[block] > i_cut) break;                                    \
            if (block) {                                                       \
                inner *= transfer[block - 1];                                  \
                prev *= transfer[block - 1];                                   \
            }                                                                  \
            long lo = cuts[block] > 1 ? cuts[block] : 1;                       \
            long hi = cuts[block + 1] < i_cut + 1 ? cuts[block + 1] : i_cut + 1; \
            for (long i = lo; i < hi; ++i) {                                   \
                double a = (DENS(i)) * rk[i];                                  \
                inner += .5 * (a + prev) * (r[i] - r[i - 1]);                  \
                y[i] = (inner * inverse[i] + rk[i] * y[i]);                    \
                prev = a;                                                      \
            }                                                                  \
        }                                                                      \
    } while (0)

void oracle_grid_yk_rho(const double *rho, const double *r, long n, const double *rk, const double *inverse,
                        const long *cuts, long ncuts, const double *transfer, long i_cut, double *y)
{
#define RHO_AT(i) rho[(i)]
    GRID_SCAN(RHO_AT);
#undef RHO_AT
}

void oracle_grid_pair_yk(const double *Pa, const double *Qa, const double *Pb, const double *Qb, const double *r,
                         long n, const double *rk, const double *inverse, const long *cuts, long ncuts,
                         const double *transfer, long i_cut, double *y)
{
#define PAIR_AT(i) (Pa[(i)] * Pb[(i)] + Qa[(i)] * Qb[(i)])
    GRID_SCAN(PAIR_AT);
#undef PAIR_AT
}

double oracle_grid_slater_rk(const double *Pa, const double *Qa, const double *Pb, const double *Qb,
                             const double *Pc, const double *Qc, const double *Pd, const double *Qd,
                             const double *r, long n, const double *rk, const double *inverse, const long *cuts,
                             long ncuts, const double *transfer, double *work)
{
    long i_cut = 0;
    for (long i = n - 1; i >= 0; --i) {
        if (Pa[i] * Pc[i] + Qa[i] * Qc[i] != 0.0) {
            i_cut = i + 1 < n - 1 ? i + 1 : n - 1;
            break;
        }
    }
    oracle_grid_pair_yk(Pb, Qb, Pd, Qd, r, n, rk, inverse, cuts, ncuts, transfer, i_cut, work);
    double prev = (Pa[0] * Pc[0] + Qa[0] * Qc[0]) * work[0];
    double total = 0.0;
    for (long i = 1; i <= i_cut; ++i) {
        double g = (Pa[i] * Pc[i] + Qa[i] * Qc[i]) * work[i];
        total += .5 * (g + prev) * (r[i] - r[i - 1]);
        prev = g;
    }
    return total;
}

struct grid_batch_ctx {
    const double *PA, *QA, *PB, *QB; long ld;
    const long *rows_a, *rows_b, *rows_k; const unsigned char *rows_ok;
    const double *RhoA; long rho_ld; const long *cons_ptr, *cons_rho;
    const double *r; long n; const double *RK, *inverse; const long *cuts; long ncuts;
    const double *transfers; long ntr; long i_cut; double *val;
};

static void grid_batch_range(void *vctx, long lo, long hi)
{
    struct grid_batch_ctx *c = (struct grid_batch_ctx *)vctx;
    double *y = (double *)malloc(sizeof(double) * (size_t)(c->i_cut + 1 > c->n ? c->i_cut + 1 : c->n));
    for (long m = lo; m < hi; ++m) {
        long s0 = c->cons_ptr[m], s1 = c->cons_ptr[m + 1];
        if (!c->rows_ok[m] || s0 == s1) continue;
        long ia = c->rows_a[m], ib = c->rows_b[m], k = c->rows_k[m];
        oracle_grid_pair_yk(c->PA + ia * c->ld, c->QA + ia * c->ld, c->PB + ib * c->ld, c->QB + ib * c->ld, c->r,
                            c->n, c->RK + k * c->n, c->inverse + k * c->n, c->cuts, c->ncuts,
                            c->transfers + k * c->ntr, c->i_cut, y);
        for (long s = s0; s < s1; ++s) {
            double total = 0.0;
            const double *w = c->RhoA + c->cons_rho[s] * c->rho_ld;
            for (long i = 0; i <= c->i_cut; ++i) total += w[i] * y[i];
            c->val[s] = total;
        }
    }
    free(y);
}

void oracle_grid_pair_dot_batch(const double *PA, const double *QA, const double *PB, const double *QB, long ld,
                                const long *rows_a, const long *rows_b, const long *rows_k,
                                const unsigned char *rows_ok, long nrows, const double *RhoA, long rho_ld,
                                const long *cons_ptr, const long *cons_rho, const double *r, long n,
                                const double *RK, const double *inverse, const long *cuts, long ncuts,
                                const double *transfers, long ntr, long i_cut, double *val, int threads)
{
    struct grid_batch_ctx ctx = {PA, QA, PB, QB, ld, rows_a, rows_b, rows_k, rows_ok, RhoA, rho_ld, cons_ptr,
                                 cons_rho, r, n, RK, inverse, cuts, ncuts, transfers, ntr, i_cut, val};
    parallel_for(grid_batch_range, &ctx, nrows, threads);
}

/* ------------------------------------------------------------------------
 * Direct potential of the Dirac-Fock driver (atomx methods/dirac_fock.py:
 * 931-967): the occupied density and the B-spline matrix of a weighted
 * function (numerics/bspline/integrals.py:18-56 _assemble_integral).
 * ---------------------------------------------------------------------- */

/* rho[i] = sum_o occ[o] * (P[o][i]^2 + Q[o][i]^2), orbital by orbital as
 * numpy's `rho_total += occ * (fP ** 2 + fQ ** 2)`; then minus the target's
 * own P^2 + Q^2 (dirac_fock.py:939-952) when target >= 0. */
void oracle_occupied_density(const double *P, const double *Q, long ld, long n_orb, const double *occ,
                             long target, long n, double *rho)
{
    for (long i = 0; i < n; ++i) {
        double acc = 0.0;
        for (long o = 0; o < n_orb; ++o) {
            const double p = P[o * ld + i], q = Q[o * ld + i];
            acc += occ[o] * (p * p + q * q);
        }
        if (target >= 0) {
            const double p = P[target * ld + i], q = Q[target * ld + i];
            acc -= p * p + q * q;
        }
        rho[i] = acc;
    }
}

/* mat (mm x mm, zeroed here) += the reference's cell loop: for each cell iv,
 * basis pair (i, j) with gi = iv+i, gj = iv+j < mm, s = sum_m
 * weights[iv][m] * b1[iv][m][i] * b2[iv][m][j]; then 0.5 * (mat + mat^T) as
 * dirac_fock.py:960/965 does. */
void oracle_bspline_sym_matrix(const double *b1, int ks1, const double *b2, int ks2, int nv, int ng,
                               const double *weights, long mm, double *out)
{
    double *mat = calloc((size_t)(mm * mm), sizeof(double));
    for (int iv = 0; iv < nv; ++iv)
        for (int i = 0; i < ks1; ++i) {
            const long gi = iv + i;
            if (gi >= mm) continue;
            for (int j = 0; j < ks2; ++j) {
                const long gj = iv + j;
                if (gj >= mm) continue;
                double s = 0.0;
                for (int m = 0; m < ng; ++m) {
                    const long node = (long)iv * ng + m;
                    s += weights[node] * b1[node * ks1 + i] * b2[node * ks2 + j];
                }
                mat[gi * mm + gj] += s;
            }
        }
    for (long a = 0; a < mm; ++a)
        for (long b = 0; b < mm; ++b) out[a * mm + b] = 0.5 * (mat[a * mm + b] + mat[b * mm + a]);
    free(mat);
}

/* Non-local exchange matrix K^k (atomx numerics/bspline/slater_yk.py:34-122,
 * _exchange_matrix_kernel), restated loop by loop: r^k and r^-(k+1) by the
 * integer power, integrand = (w fb) B_s, per column n the product density
 * fb B_n on its cells, rectangle-rule outward/inward cumulative sums over
 * the whole grid, Y^k = r^-(k+1) I_out + r^k I_in, then K[m][n] += sum_g
 * integrand Y^k cell by cell.  fb (nv*ng), bsp (nv, ng, ks), K (ns x ns). */
void oracle_exchange_matrix(const double *fb, const double *bsp, const double *gr, const double *grw, int nv,
                            int ng, int ks, int ns, int k, double *K)
{
    const long n = (long)nv * ng;
    double *rk = malloc(sizeof(double) * n), *rkm = malloc(sizeof(double) * n);
    double *integ = malloc(sizeof(double) * n * ks), *rho = malloc(sizeof(double) * n);
    double *iout = malloc(sizeof(double) * n), *iin = malloc(sizeof(double) * n), *yk = malloc(sizeof(double) * n);
    memset(K, 0, sizeof(double) * (size_t)ns * ns);
    for (long i = 0; i < n; ++i) {
        rk[i] = oracle_int_pow(gr[i], k);
        rkm[i] = oracle_int_pow(gr[i], -(long)(k + 1));
    }
    for (long i = 0; i < n; ++i) {
        const double wfb = grw[i] * fb[i];
        for (int s = 0; s < ks; ++s) integ[i * ks + s] = wfb * bsp[i * ks + s];
    }
    for (int nn = 0; nn < ns; ++nn) {
        for (long i = 0; i < n; ++i) rho[i] = 0.0;
        int lo = nn - ks + 1 < 0 ? 0 : nn - ks + 1, hi = nn + 1 > nv ? nv : nn + 1;
        for (int iv = lo; iv < hi; ++iv)
            for (int g = 0; g < ng; ++g) {
                const long idx = (long)iv * ng + g;
                rho[idx] = fb[idx] * bsp[idx * ks + (nn - iv)];
            }
        double s = 0.0;
        for (long i = 0; i < n; ++i) {
            s += grw[i] * rho[i] * rk[i];
            iout[i] = s;
        }
        s = 0.0;
        for (long i = n - 1; i >= 0; --i) {
            s += grw[i] * rho[i] * rkm[i];
            iin[i] = s;
        }
        for (long i = 0; i < n; ++i) yk[i] = rkm[i] * iout[i] + rk[i] * iin[i];
        for (int iv = 0; iv < nv; ++iv)
            for (int sidx = 0; sidx < ks; ++sidx) {
                const int m = iv + sidx;
                if (m < ns) {
                    double acc = 0.0;
                    for (int g = 0; g < ng; ++g) acc += integ[((long)iv * ng + g) * ks + sidx] * yk[(long)iv * ng + g];
                    K[(long)m * ns + nn] += acc;
                }
            }
    }
    free(rk), free(rkm), free(integ), free(rho), free(iout), free(iin), free(yk);
}
