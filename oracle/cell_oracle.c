/*
 * CPU oracle for the cell (bank) R^k engine — TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of atomx's cell algorithm (src/atomx/numerics/bspline/
 * convol.py), used by the test-suite as the checker of the device cell engine.
 * Nothing in the shipped engine links or calls it.  Every loop keeps the
 * reference's operation order, and the file is compiled with
 * -ffp-contract=off, so that with identical inputs the results agree with the
 * reference to the last bit wherever the reference itself runs without
 * fastmath.
 *
 * Restated functions (atomx, path relative to its project root):
 *   oracle_gl01              <- convol.py:253-293  (_gauss_legendre_01)
 *   oracle_bsplvb            <- convol.py:296-317  (_bsplvb_inplace)
 *   oracle_cell_moments      <- convol.py:58-94    (_compute_moments_sym)
 *   oracle_cell_triang       <- convol.py:136-250  (_triang_sym) and
 *                               convol.py:388-530  (_triang_pqpq)
 *   oracle_cell_assemble     <- convol.py:324-381  (_assemble_rkb_sym) and
 *                               convol.py:533-576  (_assemble_rkb_pqpq)
 *   oracle_density_sym       <- convol.py:713-754  (_density_sym)
 *   oracle_convol_case2      <- convol.py:853-875 / 1311-1346
 *                               (_convol_case2, _convol_case2_mixed)
 *   oracle_sum_amb_banded    <- convol.py:1349-1357 (_sum_amb_banded)
 *   oracle_convol_case1_t    <- convol.py:972-998  (_convol_case1_t)
 *   oracle_convol_case4_t    <- convol.py:1001-1059 (_convol_case4_t)
 *   oracle_rkb_bilinear      <- convol.py:1901-1942 (_rkb_bilinear)
 *
 * Layouts (C order, doubles): moments (kk, nv) with kk = ks (ks+1) / 2 packed
 * upper pairs; diagonal cells (kk_left, kk_right, nv); banks
 * rkb[i][j][ip][jp] of shape (ns, ns, ks_left, ks_right); banded densities
 * (ns, ks).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

static double ipow(double x, long n) /* Numba's float ** int: square and multiply */
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

void oracle_gl01(int n, double *x, double *w)
{
    if (n == 1) {
        x[0] = 0.5;
        w[0] = 1.0;
        return;
    }
    for (int i = 0; i < n; ++i) {
        double xi = cos(M_PI * (i + 0.75) / (n + 0.5));
        double p0 = 1.0, p1 = xi, dp = 0.0;
        for (int it = 0; it < 50; ++it) {
            p0 = 1.0;
            p1 = xi;
            for (int j = 2; j <= n; ++j) {
                double p2 = ((2 * j - 1) * xi * p1 - (j - 1) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (xi * p1 - p0) / (xi * xi - 1.0);
            double dx = p1 / dp;
            xi -= dx;
            if (fabs(dx) < 1e-15) break;
        }
        x[i] = 0.5 * (xi + 1.0);
        w[i] = 1.0 / ((1.0 - xi * xi) * dp * dp);
    }
}

void oracle_bsplvb(const double *t, int ks, double x, int left, double *b)
{
    double dr[64], dl[64];
    b[0] = 1.0;
    for (int i = 1; i < ks; ++i) b[i] = 0.0;
    for (int j = 1; j < ks; ++j) {
        dr[j] = t[left + j] - x;
        dl[j] = x - t[left + 1 - j];
        double saved = 0.0;
        for (int r = 0; r < j; ++r) {
            double term = b[r] / (dr[r + 1] + dl[j - r]);
            b[r] = saved + dr[r + 1] * term;
            saved = dl[j - r] * term;
        }
        b[j] = saved;
    }
}

/* weight of a node for the power k: w r^k, w / r^-k or w */
static double power_weight(double w, double r, int k)
{
    if (k > 0) return w * ipow(r, k);
    if (k < 0) return w / ipow(r, -k);
    return w;
}

void oracle_cell_moments(const double *bsp, const double *gr, const double *grw, int nv, int ng, int ks, int k,
                         double *rkm)
{
    double gw[64];
    for (int iv = 0; iv < nv; ++iv) {
        for (int m = 0; m < ng; ++m) gw[m] = power_weight(grw[iv * ng + m], gr[iv * ng + m], k);
        int ii = 0;
        for (int i = 0; i < ks; ++i)
            for (int j = i; j < ks; ++j) {
                double s = 0.0;
                for (int m = 0; m < ng; ++m)
                    s += bsp[((long)iv * ng + m) * ks + i] * bsp[((long)iv * ng + m) * ks + j] * gw[m];
                rkm[(long)ii * nv + iv] = s;
                ++ii;
            }
    }
}

/* INTP[(j,jp) packed][m] = int_{xbase}^{gr[iv,m]} B_j B_jp r^k over the cell of
 * knot sequence t (order ks, left = ks - 1 + iv) with n_sub GL points. */
static void inner_integrals(const double *t, int ks, int iv, const double *gr, int ng, int k, int n_sub,
                            const double *x01, const double *w01, double *intp /* (kk, ng) */)
{
    const int kk = ks * (ks + 1) / 2;
    const int left = ks - 1 + iv;
    const double xbase = t[left];
    double bsub[64][32], gwr[64];
    for (int m = 0; m < ng; ++m) {
        const double span = gr[iv * ng + m] - xbase;
        if (span < 1e-30) {
            for (int p = 0; p < kk; ++p) intp[p * ng + m] = 0.0;
            continue;
        }
        for (int n = 0; n < n_sub; ++n) {
            const double gx = xbase + span * x01[n];
            oracle_bsplvb(t, ks, gx, left, bsub[n]);
            const double w = span * w01[n];
            gwr[n] = k > 0 ? w * ipow(gx, k) : (k < 0 ? w / ipow(gx, -k) : w);
        }
        int p = 0;
        for (int j = 0; j < ks; ++j)
            for (int jp = j; jp < ks; ++jp) {
                double s = 0.0;
                for (int n = 0; n < n_sub; ++n) s += bsub[n][j] * bsub[n][jp] * gwr[n];
                intp[p * ng + m] = s;
                ++p;
            }
    }
}

/* a[ii][jj] = sum_m B_i B_ip(outer, m) grw / r^(k+1) * INTP[jj][m] */
static void outer_sum(const double *bsp_o, int ks_o, int iv, const double *gr, const double *grw, int ng, int k,
                      const double *intp, int kk_in, double *a /* (kk_o, kk_in) */, int transpose)
{
    double ow[64], bw[64];
    for (int m = 0; m < ng; ++m) ow[m] = grw[iv * ng + m] / ipow(gr[iv * ng + m], k + 1);
    const int kk_o = ks_o * (ks_o + 1) / 2;
    int ii = 0;
    for (int i = 0; i < ks_o; ++i)
        for (int ip = i; ip < ks_o; ++ip) {
            for (int m = 0; m < ng; ++m)
                bw[m] = bsp_o[((long)iv * ng + m) * ks_o + i] * bsp_o[((long)iv * ng + m) * ks_o + ip] * ow[m];
            for (int jj = 0; jj < kk_in; ++jj) {
                double s = 0.0;
                for (int m = 0; m < ng; ++m) s += bw[m] * intp[jj * ng + m];
                if (transpose) a[(long)jj * kk_o + ii] = s;
                else a[(long)ii * kk_in + jj] = s;
            }
            ++ii;
        }
}

/* Diagonal cells.  Same component (bsp_l == bsp_r, t_l == t_r): _triang_sym
 * with n_sub = ks + k/2 and rkd = a + a^T.  Different components:
 * _triang_pqpq (left outer with right inner, plus right outer with left inner)
 * with n_sub = max(ks_l, ks_r) + k/2.  Output (kk_l, kk_r, nv). */
void oracle_cell_triang(const double *bsp_l, const double *bsp_r, const double *gr, const double *grw,
                        const double *t_l, const double *t_r, int nv, int ng, int ks_l, int ks_r, int same, int k,
                        double *rkd)
{
    const int kkl = ks_l * (ks_l + 1) / 2, kkr = ks_r * (ks_r + 1) / 2;
    const int n_sub = (same ? ks_l : (ks_l > ks_r ? ks_l : ks_r)) + (k >= 0 ? k / 2 : 0);
    double x01[64], w01[64];
    oracle_gl01(n_sub, x01, w01);
    double *intp_r = malloc(sizeof(double) * kkr * ng), *intp_l = malloc(sizeof(double) * kkl * ng);
    double *a = malloc(sizeof(double) * kkl * kkr), *at = malloc(sizeof(double) * kkl * kkr);
    for (int iv = 0; iv < nv; ++iv) {
        inner_integrals(t_r, ks_r, iv, gr, ng, k, n_sub, x01, w01, intp_r);
        outer_sum(bsp_l, ks_l, iv, gr, grw, ng, k, intp_r, kkr, a, 0);
        if (same) {
            for (int ii = 0; ii < kkl; ++ii)
                for (int jj = 0; jj < kkr; ++jj)
                    rkd[((long)ii * kkr + jj) * nv + iv] = a[ii * kkr + jj] + a[jj * kkr + ii];
        } else {
            inner_integrals(t_l, ks_l, iv, gr, ng, k, n_sub, x01, w01, intp_l);
            outer_sum(bsp_r, ks_r, iv, gr, grw, ng, k, intp_l, kkl, at, 1);
            for (int ii = 0; ii < kkl; ++ii)
                for (int jj = 0; jj < kkr; ++jj)
                    rkd[((long)ii * kkr + jj) * nv + iv] = a[ii * kkr + jj] + at[ii * kkr + jj];
        }
    }
    free(intp_r); free(intp_l); free(a); free(at);
}

/* Bank assembly: rkb[i][j][ip][jp] (ns, ns, ks_l, ks_r) from the local moments
 * of the left (rising_l r^k, falling_l r^-(k+1)) and right components and the
 * diagonal cells; cells iv < jv give rising_l[ii][iv] falling_r[jj][jv], cells
 * iv > jv give rising_r[jj][jv] falling_l[ii][iv].  Contributions to one
 * element arrive in the reference's order (jv, then iv, ascending). */
void oracle_cell_assemble(const double *rising_l, const double *falling_l, const double *rising_r,
                          const double *falling_r, const double *diag, int nv, int ks_l, int ks_r, int ns,
                          double *rkb)
{
    const int kkr = ks_r * (ks_r + 1) / 2;
    memset(rkb, 0, sizeof(double) * (size_t)ns * ns * ks_l * ks_r);
    for (int jv = 0; jv < nv; ++jv) {
        int jj = 0;
        for (int jh = 0; jh < ks_r; ++jh)
            for (int jhp = jh; jhp < ks_r; ++jhp, ++jj) {
                const int j = jv + jh, jp = jhp - jh;
                for (int iv = 0; iv < nv; ++iv) {
                    int ii = 0;
                    for (int ih = 0; ih < ks_l; ++ih)
                        for (int ihp = ih; ihp < ks_l; ++ihp, ++ii) {
                            const int i = iv + ih, ip = ihp - ih;
                            double c;
                            if (iv < jv) c = rising_l[(long)ii * nv + iv] * falling_r[(long)jj * nv + jv];
                            else if (iv > jv) c = rising_r[(long)jj * nv + jv] * falling_l[(long)ii * nv + iv];
                            else c = diag[((long)ii * kkr + jj) * nv + iv];
                            if (i < ns && j < ns) rkb[(((long)i * ns + j) * ks_l + ip) * ks_r + jp] += c;
                        }
                }
            }
    }
}

void oracle_density_sym(const double *p1, int n1, const double *p2, int n2, int ns, int ks, double *d)
{
    memset(d, 0, sizeof(double) * (size_t)ns * ks);
    const int lim = n1 < ns ? n1 : ns;
    for (int i = 0; i < lim; ++i) {
        if (i < n2) d[i * ks] = p1[i] * p2[i];
        for (int s = 1; s < ks; ++s) {
            const int ip = i + s;
            if (ip >= ns) break;
            double v = 0.0;
            if (ip < n2) v += p1[i] * p2[ip];
            if (ip < n1 && i < n2) v += p1[ip] * p2[i];
            d[i * ks + s] = v;
        }
    }
}

/* a[j][jp] = sum_ip sum_i rkb[i][j][ip][jp] d_left[i][ip] over i + ip < n_left,
 * for the (ns_c, ks_r) output band with j + jp < ns_c; the bank is
 * (ns_bank, ns_bank, ks_l, ks_r).  _convol_case2 is n_left = ns_c. */
void oracle_convol_case2(const double *rkb, int ns_bank, const double *d_left, int n_left, int ns_c, int ks_l,
                         int ks_r, double *a)
{
    for (int idx = 0; idx < ns_c * ks_r; ++idx) {
        const int j = idx / ks_r, jp = idx % ks_r;
        double s = 0.0;
        if (j + jp < ns_c)
            for (int ip = 0; ip < ks_l; ++ip)
                for (int i = 0; i < n_left; ++i) {
                    if (i + ip >= n_left) continue;
                    s += rkb[(((long)i * ns_bank + j) * ks_l + ip) * ks_r + jp] * d_left[i * ks_l + ip];
                }
        a[idx] = s;
    }
}

double oracle_sum_amb_banded(const double *a, const double *b, int ns, int ks)
{
    double s = 0.0;
    for (int ip = 0; ip < ks; ++ip)
        for (int i = 0; i < ns; ++i)
            if (i + ip < ns) s += a[i * ks + ip] * b[i * ks + ip];
    return s;
}

/* a[i][ip] = sum_jp sum_j rkb[i][j][ip][jp] d[j][jp] over j < ns - jp
 * (the reference runs this one with fastmath; here in plain order). */
void oracle_convol_case1(const double *rkb, const double *d, int ns, int ks_l, int ks_r, double *a)
{
    memset(a, 0, sizeof(double) * (size_t)ns * ks_l);
    for (int ip = 0; ip < ks_l; ++ip)
        for (int i = 0; i < ns - ip; ++i) {
            double s = 0.0;
            for (int jp = 0; jp < ks_r; ++jp)
                for (int j = 0; j < ns - jp; ++j) s += rkb[(((long)i * ns + j) * ks_l + ip) * ks_r + jp] * d[j * ks_r + jp];
            a[i * ks_l + ip] = s;
        }
}

/* Exchange contraction on the full density d (ns x ns): the four families of
 * _convol_case4_t in its order; symmetric = compute the lower triangle and
 * mirror it. */
void oracle_convol_case4(const double *rkb, const double *d, int ns, int ks, int ks_r, int symmetric, double *a)
{
#define RKB(i, j, ip, jp) rkb[(((long)(i) * ns + (j)) * ks + (ip)) * ks_r + (jp)]
    memset(a, 0, sizeof(double) * (size_t)ns * ns);
    for (int row = 0; row < ns; ++row) {
        double *buf = a + (long)row * ns;
        const int col_limit = symmetric ? row + 1 : ns;
        for (int ip = 0; ip < ks; ++ip) {
            const int i = row - ip;
            if (i < 0) continue;
            for (int jp = 0; jp < ks_r; ++jp) {
                const int lim = ns - jp < col_limit ? ns - jp : col_limit;
                for (int col = 0; col < lim; ++col) buf[col] += RKB(i, col, ip, jp) * d[(long)i * ns + col + jp];
            }
        }
        for (int ip = 1; ip < ks; ++ip) {
            const int ii = row + ip;
            if (ii >= ns) continue;
            for (int jp = 0; jp < ks_r; ++jp) {
                const int lim = ns - jp < col_limit ? ns - jp : col_limit;
                for (int col = 0; col < lim; ++col) buf[col] += RKB(row, col, ip, jp) * d[(long)ii * ns + col + jp];
            }
        }
        for (int jp = 1; jp < ks_r; ++jp)
            for (int ip = 0; ip < ks; ++ip) {
                const int i = row - ip;
                if (i < 0) continue;
                for (int col = jp; col < col_limit; ++col)
                    buf[col] += RKB(i, col - jp, ip, jp) * d[(long)i * ns + col - jp];
            }
        for (int ip = 1; ip < ks; ++ip) {
            const int ii = row + ip;
            if (ii >= ns) continue;
            for (int jp = 1; jp < ks_r; ++jp)
                for (int col = jp; col < col_limit; ++col)
                    buf[col] += RKB(row, col - jp, ip, jp) * d[(long)ii * ns + col - jp];
        }
        if (symmetric)
            for (int col = 0; col < row; ++col) a[(long)col * ns + row] = buf[col];
    }
#undef RKB
}

/* M[m][n] = sum rkb[i][j][ip][jp] sigma_wa(i, ip; m) sigma_wb(j, jp; n) over
 * i + ip < n_left, j + jp < n_right; M is (ns_out, ns_out). */
void oracle_rkb_bilinear(const double *rkb, int ns_bank, const double *wa, const double *wb, int n_left,
                         int n_right, int ks_l, int ks_r, int ns_out, double *M)
{
    double *T = calloc((size_t)ns_out * n_right * ks_r, sizeof(double));
    for (int i = 0; i < n_left; ++i)
        for (int j = 0; j < n_right; ++j)
            for (int ip = 0; ip < ks_l; ++ip) {
                if (i + ip >= n_left) break;
                const double wi = wa[i], wip = wa[i + ip];
                for (int jp = 0; jp < ks_r; ++jp) {
                    if (j + jp >= n_right) break;
                    const double c = rkb[(((long)i * ns_bank + j) * ks_l + ip) * ks_r + jp];
                    T[((long)i * n_right + j) * ks_r + jp] += c * wip;
                    if (ip > 0) T[((long)(i + ip) * n_right + j) * ks_r + jp] += c * wi;
                }
            }
    memset(M, 0, sizeof(double) * (size_t)ns_out * ns_out);
    for (int m = 0; m < ns_out; ++m)
        for (int j = 0; j < n_right; ++j) {
            const double wj = wb[j];
            for (int jp = 0; jp < ks_r; ++jp) {
                if (j + jp >= n_right) break;
                const double t = T[((long)m * n_right + j) * ks_r + jp];
                M[(long)m * ns_out + j] += t * wb[j + jp];
                if (jp > 0) M[(long)m * ns_out + j + jp] += t * wj;
            }
        }
    free(T);
}
