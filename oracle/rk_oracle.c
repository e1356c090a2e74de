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
 *       integral.
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
