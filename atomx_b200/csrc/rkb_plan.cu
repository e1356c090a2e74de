// Host-side planning for the split engine: the factored Green operator of one
// multipole on one grid, packed as the device kernels read it.
//
// With u = r^-(k+1), v = r^k per node and the interpolatory partial matrices
// mo, mi (mo + mi = 1) of the cell rule, atomx's Y^k (numerics/yk.py:88-154)
// contracts to R = g^T G g with G's cell blocks u_i v_j mo_ij + v_i u_j mi_ij
// (diagonal cells) and rank-one kernel samples off the diagonal.  The body
// (cells >= 1) gets the structured modified Cholesky
//     S_m = D_m - sigma u_m u_m^T,   L_m L_m^T = S_m + Delta_m,
//     c_m = L_m^-1 (v_m - sigma u_m),  sigma += |c_m|^2,
// where Delta_m = sum_e z_e z_e^T lifts every eigenvalue of the diagonally
// scaled S_m below tau * lambda_max to max(|lambda|, tau lambda_max); the z_e
// become the negative-sign columns Z.  The core cell 0 stays in FP64: its
// block G_00 and the rank-one core-body coupling v_0 u_b^T, which the row
// kernels carry as the two scaled moments alpha*sx = sx v_0.g_0 and
// q/sx = u_b.g_b / sx.  sx = r_b^-(k+1)/2 r_l^-k/2 (r_l the last core node,
// r_b the first body node) bounds both by |g|_1 / sqrt(r_b).  This is the
// same factorisation as atomx_b200.split_plan.green_factor (numpy); the
// eigenproblems here are solved by cyclic Jacobi rotations (ng <= 32), so
// eigenvector signs may differ, which leaves every z_e z_e^T and the factor
// unchanged.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "rkb_common.cuh"

namespace rkb {
namespace plan {

// Symmetric eigenproblem A = V diag(w) V^T (n <= 32) by cyclic Jacobi.
// A is overwritten; V is row-major with eigenvectors in columns.
static void jacobi_eigh(int n, double *A, double *w, double *V) {
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) V[i * n + j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < n; ++i) {
            diag += A[i * n + i] * A[i * n + i];
            for (int j = i + 1; j < n; ++j) off += A[i * n + j] * A[i * n + j];
        }
        if (off <= 1e-34 * diag || off == 0.0) break;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[p * n + q];
                if (apq == 0.0) continue;
                const double app = A[p * n + p], aqq = A[q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int i = 0; i < n; ++i) {  // A <- A J (columns p, q)
                    const double aip = A[i * n + p], aiq = A[i * n + q];
                    A[i * n + p] = c * aip - s * aiq;
                    A[i * n + q] = s * aip + c * aiq;
                }
                for (int j = 0; j < n; ++j) {  // A <- J^T A (rows p, q)
                    const double apj = A[p * n + j], aqj = A[q * n + j];
                    A[p * n + j] = c * apj - s * aqj;
                    A[q * n + j] = s * apj + c * aqj;
                }
                for (int i = 0; i < n; ++i) {  // V <- V J
                    const double vip = V[i * n + p], viq = V[i * n + q];
                    V[i * n + p] = c * vip - s * viq;
                    V[i * n + q] = s * vip + c * viq;
                }
            }
        }
    }
    for (int i = 0; i < n; ++i) w[i] = A[i * n + i];
}

// Lower Cholesky factor of an SPD matrix (row-major, in place below the
// diagonal; the strict upper part is zeroed).  False if not positive.
static bool cholesky(int n, double *A) {
    for (int j = 0; j < n; ++j) {
        double d = A[j * n + j];
        for (int p = 0; p < j; ++p) d -= A[j * n + p] * A[j * n + p];
        if (!(d > 0.0)) return false;
        d = std::sqrt(d);
        A[j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double s = A[i * n + j];
            for (int p = 0; p < j; ++p) s -= A[i * n + p] * A[j * n + p];
            A[i * n + j] = s / d;
        }
        for (int i = 0; i < j; ++i) A[i * n + j] = 0.0;
    }
    return true;
}

// x = L^-1 b (forward substitution, L lower, row-major).
static void lower_solve(int n, const double *L, const double *b, double *x) {
    for (int i = 0; i < n; ++i) {
        double s = b[i];
        for (int p = 0; p < i; ++p) s -= L[i * n + p] * x[p];
        x[i] = s / L[i * n + i];
    }
}

}  // namespace plan
}  // namespace rkb

using namespace rkb;

extern "C" long rkb_green_factor(const double *r, int nv, int ng, int k, double tau, const double *mo,
                                 const double *mi, double *out, long cap) {
    RKB_CHECK_ARG(r != nullptr && mo != nullptr && mi != nullptr && out != nullptr, "null argument");
    RKB_CHECK_ARG(nv >= 2 && ng >= 1 && ng <= RKB_MAX_NG, "invalid grid (nv=%d, ng=%d)", nv, ng);
    RKB_CHECK_ARG(k >= 0 && tau >= 0.0, "invalid multipole or shift threshold");
    const int n = nv * ng, g2 = ng * ng;
    const long fixed = (long)n + (long)nv * g2 + (long)nv * ng + ng + g2 + 2;
    RKB_CHECK_ARG(cap >= fixed, "output capacity %ld below the %ld fixed doubles", cap, fixed);
    std::vector<double> u(n), v(n), Lb((size_t)nv * g2, 0.0), C((size_t)nv * ng, 0.0);
    for (int i = 0; i < n; ++i) {
        u[i] = std::pow(r[i], -(double)(k + 1));
        v[i] = std::pow(r[i], (double)k);
    }
    std::vector<double> D(g2), S(g2), A(g2), T(g2), V(g2), w(ng), d(ng), rhs(ng);
    std::vector<int> zcell;
    std::vector<double> zvec;
    double sigma = 0.0;
    for (int m = 1; m < nv; ++m) {
        const double *um = &u[(size_t)m * ng], *vm = &v[(size_t)m * ng];
        for (int i = 0; i < ng; ++i)
            for (int j = 0; j < ng; ++j)
                D[i * ng + j] = um[i] * vm[j] * mo[i * ng + j] + vm[i] * um[j] * mi[i * ng + j];
        for (int i = 0; i < ng; ++i)
            for (int j = 0; j < i; ++j) {
                const double s = 0.5 * (D[i * ng + j] + D[j * ng + i]);
                D[i * ng + j] = D[j * ng + i] = s;
            }
        for (int i = 0; i < ng; ++i) d[i] = std::sqrt(std::fabs(D[i * ng + i]));
        for (int i = 0; i < ng; ++i)
            for (int j = 0; j < ng; ++j) {
                S[i * ng + j] = D[i * ng + j] - sigma * um[i] * um[j];
                A[i * ng + j] = S[i * ng + j] / (d[i] * d[j]);
            }
        // Certificate that no eigenvalue needs a shift: with lambda_max <= gb
        // (Gershgorin), a Cholesky of A - tau*gb*I proves lambda_min > tau*gb
        // >= tau*lambda_max, and the eigensolve is skipped (most cells).
        double gb = 0.0;
        for (int i = 0; i < ng; ++i) {
            double row = 0.0;
            for (int j = 0; j < ng; ++j) row += std::fabs(A[i * ng + j]);
            gb = std::fmax(gb, row);
        }
        std::memcpy(T.data(), A.data(), sizeof(double) * g2);
        for (int i = 0; i < ng; ++i) T[i * ng + i] -= tau * gb;
        const bool no_shift = tau > 0.0 && plan::cholesky(ng, T.data());
        if (!no_shift) plan::jacobi_eigh(ng, A.data(), w.data(), V.data());
        double lmax = no_shift ? 0.0 : w[0];
        for (int e = 1; e < ng && !no_shift; ++e) lmax = std::fmax(lmax, w[e]);
        const double floor = tau * lmax;
        for (int e = 0; e < ng && !no_shift; ++e) {
            if (!(w[e] < floor)) continue;
            const double shift = std::fmax(std::fabs(w[e]), floor) - w[e];
            const double sq = std::sqrt(shift);
            zcell.push_back(m);
            const size_t z0 = zvec.size();
            for (int i = 0; i < ng; ++i) zvec.push_back(sq * V[i * ng + e] * d[i]);
            for (int i = 0; i < ng; ++i)
                for (int j = 0; j < ng; ++j) S[i * ng + j] += zvec[z0 + i] * zvec[z0 + j];
        }
        double *Lm = &Lb[(size_t)m * g2];
        std::memcpy(Lm, S.data(), sizeof(double) * g2);
        if (!plan::cholesky(ng, Lm)) {
            set_error("green factor: cell %d of multipole %d is not positive after the shift", m, k);
            return -(long)RKB_ENONFINITE;
        }
        for (int i = 0; i < ng; ++i) rhs[i] = vm[i] - sigma * um[i];
        double *Cm = &C[(size_t)m * ng];
        plan::lower_solve(ng, Lm, rhs.data(), Cm);
        for (int i = 0; i < ng; ++i) sigma += Cm[i] * Cm[i];
    }
    const long nz = (long)zcell.size();
    const long total = fixed + nz * (ng + 1);
    RKB_CHECK_ARG(cap >= total, "output capacity %ld below the %ld doubles of this factor", cap, total);
    // u[N] | Lb[nv][ng][ng] | C[nv][ng] | v0[ng] | G00[ng][ng] | sx | nZ | nZ x (cell, z[ng])
    double *o = out;
    std::memcpy(o, u.data(), sizeof(double) * n); o += n;
    std::memcpy(o, Lb.data(), sizeof(double) * (size_t)nv * g2); o += (size_t)nv * g2;
    std::memcpy(o, C.data(), sizeof(double) * (size_t)nv * ng); o += (size_t)nv * ng;
    for (int i = 0; i < ng; ++i) o[i] = v[i];
    o += ng;
    for (int i = 0; i < ng; ++i)
        for (int j = 0; j < ng; ++j) o[i * ng + j] = u[i] * v[j] * mo[i * ng + j] + v[i] * u[j] * mi[i * ng + j];
    o += g2;
    *o++ = std::sqrt(u[ng]) / std::sqrt(v[ng - 1]);  // sx (k = 0: v = 1)
    *o++ = (double)nz;
    for (long e = 0; e < nz; ++e) {
        *o++ = (double)zcell[e];
        for (int i = 0; i < ng; ++i) *o++ = zvec[(size_t)e * ng + i];
    }
    return total;
}

// All multipoles' factor tables of one grid in one call: the factorisations
// (each the serial recursion of rkb_green_factor) run on up to nthreads host
// threads, one multipole per task, then the packed tables are laid end to end
// in ks order and the cell-minor copy is written beside them.  A serving
// planner gets every table of a request without the interpreter lock and
// without a transpose pass of its own.
extern "C" long rkb_green_tables(const double *r, int nv, int ng, const int *ks, int nk, double tau,
                                 const double *mo, const double *mi, int nthreads, int kmax, double *flat,
                                 long flat_cap, long *koff, double *flat_t, long flat_t_cap, long *koff_t,
                                 long *nz) {
    RKB_CHECK_ARG(r != nullptr && ks != nullptr && mo != nullptr && mi != nullptr && flat != nullptr &&
                      koff != nullptr && flat_t != nullptr && koff_t != nullptr && nz != nullptr,
                  "null argument");
    RKB_CHECK_ARG(nk >= 1 && nv >= 2 && ng >= 1 && ng <= RKB_MAX_NG, "invalid grid or multipole count");
    for (int i = 0; i < nk; ++i)
        RKB_CHECK_ARG(ks[i] >= 0 && ks[i] <= kmax && (i == 0 || ks[i] > ks[i - 1]),
                      "multipoles must be increasing and within 0..kmax (%d)", kmax);
    const int n = nv * ng, g2 = ng * ng;
    const long cap1 = (long)n + (long)nv * g2 + (long)n + ng + g2 + 2 + (long)n * (ng + 1);
    const long per_t = 2L * n + (long)nv * g2;
    std::vector<std::vector<double>> tab((size_t)nk);
    std::vector<long> got((size_t)nk, 0);
    std::vector<std::string> err((size_t)nk);
    std::atomic<int> next(0);
    auto work = [&]() {
        for (int i = next.fetch_add(1); i < nk; i = next.fetch_add(1)) {
            tab[(size_t)i].resize((size_t)cap1);
            got[(size_t)i] = rkb_green_factor(r, nv, ng, ks[i], tau, mo, mi, tab[(size_t)i].data(), cap1);
            if (got[(size_t)i] < 0) err[(size_t)i] = rkb_last_error();
        }
    };
    const int nt = std::max(1, std::min(nthreads, nk));
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto &th : pool) th.join();
    for (int i = 0; i < nk; ++i)
        if (got[(size_t)i] < 0) {
            set_error("%s", err[(size_t)i].c_str());
            return got[(size_t)i];
        }
    for (int k = 0; k <= kmax; ++k) koff[k] = koff_t[k] = -1;
    long pos = 0, pos_t = 0;
    for (int i = 0; i < nk; ++i) {
        const long len = got[(size_t)i];
        RKB_CHECK_ARG(pos + len <= flat_cap && pos_t + per_t <= flat_t_cap, "table capacity too small");
        const double *F = tab[(size_t)i].data();
        std::memcpy(flat + pos, F, sizeof(double) * (size_t)len);
        koff[ks[i]] = pos;
        nz[i] = (long)F[(long)n + (long)nv * g2 + n + ng + g2 + 1];
        // cell-minor copy: u^T[ng][nv] | C^T[ng][nv] | Lb as [ng][ng][nv]
        double *T = flat_t + pos_t;
        const double *u = F, *Lb = F + n, *C = F + n + (long)nv * g2;
        for (int m = 0; m < nv; ++m)
            for (int j = 0; j < ng; ++j) {
                T[(long)j * nv + m] = u[(long)m * ng + j];
                T[(long)n + (long)j * nv + m] = C[(long)m * ng + j];
            }
        for (int m = 0; m < nv; ++m)
            for (int a = 0; a < ng; ++a)
                for (int b = 0; b < ng; ++b)
                    T[2L * n + ((long)a * ng + b) * nv + m] = Lb[(long)m * g2 + (long)a * ng + b];
        koff_t[ks[i]] = pos_t;
        pos += len;
        pos_t += per_t;
    }
    return pos;
}

// Table plan of an orbital set, filled natively (the caller sizes it): pairs
// a <= c by kappa-shell blocks (shell pairs i <= j, i-major; inside a block
// a-major, a <= c within one shell), then the rows (pair, k) grouped by k in
// increasing order, each k's pairs ascending.
extern "C" long rkb_table_plan(const long *shell_start, const long *shell_size, int n_shells,
                               const unsigned char *allowed, int k_max, long n_pairs, long n_rows, long *pairs,
                               long *pair_block, long *row_pair, long *row_k) {
    RKB_CHECK_ARG(shell_start != nullptr && shell_size != nullptr && allowed != nullptr && pairs != nullptr &&
                      pair_block != nullptr && row_pair != nullptr && row_k != nullptr,
                  "null argument");
    RKB_CHECK_ARG(n_shells >= 1 && k_max >= 0 && n_pairs >= 0 && n_rows >= 0, "invalid plan sizes");
    const long nb = (long)n_shells * (n_shells + 1) / 2;
    std::vector<long> boff((size_t)nb + 1);
    long p = 0, b = 0;
    for (int i = 0; i < n_shells; ++i)
        for (int j = i; j < n_shells; ++j, ++b) {
            boff[(size_t)b] = p;
            const long na = shell_size[i], nc = shell_size[j], a0 = shell_start[i], c0 = shell_start[j];
            const long need = i == j ? na * (na + 1) / 2 : na * nc;
            RKB_CHECK_ARG(na >= 0 && nc >= 0 && p + need <= n_pairs, "pair count %ld exceeded", n_pairs);
            for (long a = 0; a < na; ++a)
                for (long c = (i == j ? a : 0); c < nc; ++c, ++p) {
                    pairs[2 * p] = a0 + a;
                    pairs[2 * p + 1] = c0 + c;
                    pair_block[p] = b;
                }
        }
    boff[(size_t)nb] = p;
    RKB_CHECK_ARG(p == n_pairs, "the shells give %ld pairs, not %ld", p, n_pairs);
    long q = 0;
    for (int k = 0; k <= k_max; ++k)
        for (long blk = 0; blk < nb; ++blk) {
            if (!allowed[blk * (k_max + 1) + k]) continue;
            const long s = boff[(size_t)blk], e = boff[(size_t)blk + 1];
            RKB_CHECK_ARG(q + (e - s) <= n_rows, "row count %ld exceeded", n_rows);
            for (long t = s; t < e; ++t, ++q) {
                row_pair[q] = t;
                row_k[q] = k;
            }
        }
    RKB_CHECK_ARG(q == n_rows, "the allowed multipoles give %ld rows, not %ld", q, n_rows);
    return q;
}
