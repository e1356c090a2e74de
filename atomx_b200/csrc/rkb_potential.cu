// One-electron potential matrices on the device built on Y^k: the direct
// (Hartree) potential of atomx's Dirac-Fock driver (methods/dirac_fock.py:
// 931-967, DFSolver._build_direct_potential_yk) and the non-local exchange
// matrix of numerics/bspline/slater_yk.py:34-155 (below).
//
//   rho    = sum_o occ_o (P_o^2 + Q_o^2)  [- (P_t^2 + Q_t^2) for a target orbital]
//   Y^0    = compute_yk(rho, k = 0)                      (rkb_yk_rows)
//   V_J    = sym <B_i | grw Y^0 | B_j>  for the P and the Q basis
//
// Both kernels follow the reference's order of operations exactly (the
// density accumulates orbital by orbital as numpy's `rho += occ * (fP**2 +
// fQ**2)`; the matrix element sums nodes in order and cells in increasing
// order as numerics/bspline/integrals.py:18-56 `_assemble_integral`), with
// separate multiplies and adds.
#include "rkb_common.cuh"

namespace rkb {
namespace potential {

// One thread per node.
__global__ void occupied_density_kernel(const double *__restrict__ P, const double *__restrict__ Q, long ld,
                                        long n_orb, const double *__restrict__ occ, long target, long n,
                                        double *__restrict__ rho) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc = 0.0;
    for (long o = 0; o < n_orb; ++o) {
        const double p = P[o * ld + i], q = Q[o * ld + i];
        acc = __dadd_rn(acc, __dmul_rn(occ[o], __dadd_rn(__dmul_rn(p, p), __dmul_rn(q, q))));
    }
    if (target >= 0) {
        const double p = P[target * ld + i], q = Q[target * ld + i];
        acc = __dsub_rn(acc, __dadd_rn(__dmul_rn(p, p), __dmul_rn(q, q)));
    }
    rho[i] = acc;
}

// M(gi, gj) = sum over cells iv (increasing) with 0 <= gi-iv < ks1 and
// 0 <= gj-iv < ks2 of  sum_m (wt[iv,m] * B1[iv,m,gi-iv]) * B2[iv,m,gj-iv],
// wt = w * f (or w when f is null).
__device__ double band_element(const double *__restrict__ b1, int ks1, const double *__restrict__ b2, int ks2,
                               int nv, int ng, const double *__restrict__ w, const double *__restrict__ f, long gi,
                               long gj) {
    long lo = gi - ks1 + 1;
    if (gj - ks2 + 1 > lo) lo = gj - ks2 + 1;
    if (lo < 0) lo = 0;
    long hi = gi < gj ? gi : gj;
    if (hi > nv - 1) hi = nv - 1;
    double mat = 0.0;
    for (long iv = lo; iv <= hi; ++iv) {
        const long i = gi - iv, j = gj - iv;
        double s = 0.0;
        for (int m = 0; m < ng; ++m) {
            const long node = iv * ng + m;
            const double wt = f ? __dmul_rn(w[node], f[node]) : w[node];
            s = __dadd_rn(s, __dmul_rn(__dmul_rn(wt, b1[node * ks1 + i]), b2[node * ks2 + j]));
        }
        mat = __dadd_rn(mat, s);
    }
    return mat;
}

// One thread per (gi, gj) of the mm x mm output: 0.5 * (M + M^T), zero off the band.
__global__ void sym_band_matrix_kernel(const double *__restrict__ b1, int ks1, const double *__restrict__ b2,
                                       int ks2, int nv, int ng, const double *__restrict__ w,
                                       const double *__restrict__ f, long mm, double *__restrict__ out) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mm * mm) return;
    const long gi = t / mm, gj = t - gi * mm;
    const double a = band_element(b1, ks1, b2, ks2, nv, ng, w, f, gi, gj);
    const double b = band_element(b1, ks1, b2, ks2, nv, ng, w, f, gj, gi);
    out[t] = __dmul_rn(0.5, __dadd_rn(a, b));
}

// ---------------------------------------------------------------------------
// Exchange matrix K^k_{mn} = int B_m fb Y^k[fb B_n] with rectangle-rule
// cumulative sums (atomx numerics/bspline/slater_yk.py:34-122,
// _exchange_matrix_kernel).  One block per column n.  rho_n = fb B_n is
// nonzero only on the cells [n-ks+1, n], so the outward sums are zero before
// that support and a constant after it, and the inward sums the reverse:
// thread 0 runs the two sequential sums over the support only, in the
// reference's order, then every point gets
//     Y^k_i = r_i^-(k+1) I_out(i) + r_i^k I_in(i)
// and thread m accumulates K[m][n] cell by cell and node by node as the
// reference does.  Shared memory: Y^k and w*fb for the whole row (2N doubles)
// plus the support's two partial-sum arrays (2 * ks * ng doubles).
__global__ void exchange_column_kernel(const double *__restrict__ fb, const double *__restrict__ bsp,
                                       const double *__restrict__ r, const double *__restrict__ w, int nv, int ng,
                                       int ks, int ns, int k, double *__restrict__ K) {
    extern __shared__ double sx[];
    const long N = (long)nv * ng;
    double *yk = sx, *wfb = sx + N, *iout = wfb + N, *iin = iout + (long)ks * ng;
    const int n_idx = blockIdx.x;
    const int lo = n_idx - ks + 1 < 0 ? 0 : n_idx - ks + 1;
    const int hi = n_idx + 1 > nv ? nv : n_idx + 1;  // cells [lo, hi)
    const long p0 = (long)lo * ng, p1 = (long)hi * ng;  // support points [p0, p1)
    for (long i = threadIdx.x; i < N; i += blockDim.x) wfb[i] = __dmul_rn(w[i], fb[i]);
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (long i = p0; i < p1; ++i) {
            const int iv = (int)(i / ng), ls = n_idx - iv;
            const double rho = __dmul_rn(fb[i], bsp[i * ks + ls]);
            s = __dadd_rn(s, __dmul_rn(__dmul_rn(w[i], rho), int_pow(r[i], k)));
            iout[i - p0] = s;
        }
        s = 0.0;
        for (long i = p1 - 1; i >= p0; --i) {
            const int iv = (int)(i / ng), ls = n_idx - iv;
            const double rho = __dmul_rn(fb[i], bsp[i * ks + ls]);
            s = __dadd_rn(s, __dmul_rn(__dmul_rn(w[i], rho), int_pow(r[i], -(k + 1))));
            iin[i - p0] = s;
        }
    }
    __syncthreads();
    const double c_out = p1 > p0 ? iout[p1 - p0 - 1] : 0.0, c_in = p1 > p0 ? iin[0] : 0.0;
    for (long i = threadIdx.x; i < N; i += blockDim.x) {
        const double o = i < p0 ? 0.0 : (i < p1 ? iout[i - p0] : c_out);
        const double in = i < p0 ? c_in : (i < p1 ? iin[i - p0] : 0.0);
        yk[i] = __dadd_rn(__dmul_rn(int_pow(r[i], -(k + 1)), o), __dmul_rn(int_pow(r[i], k), in));
    }
    __syncthreads();
    for (int m = threadIdx.x; m < ns; m += blockDim.x) {
        double kmn = 0.0;
        const int c0 = m - ks + 1 < 0 ? 0 : m - ks + 1, c1 = m < nv - 1 ? m : nv - 1;
        for (int iv = c0; iv <= c1; ++iv) {
            const int sidx = m - iv;
            double acc = 0.0;
            for (int g = 0; g < ng; ++g) {
                const long idx = (long)iv * ng + g;
                acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(wfb[idx], bsp[idx * ks + sidx]), yk[idx]));
            }
            kmn = __dadd_rn(kmn, acc);
        }
        K[(long)m * ns + n_idx] = kmn;
    }
}

}  // namespace potential
}  // namespace rkb

using namespace rkb;

extern "C" int rkb_exchange_matrix(const double *d_fb, const double *d_bsp, const double *d_r, const double *d_w,
                                   int nv, int ng, int ks, int ns, int k, double *d_K, void *stream) {
    RKB_CHECK_ARG(nv >= 1 && ng >= 1 && ks >= 1 && ns >= 1 && ns <= nv + ks - 1, "invalid sizes");
    RKB_CHECK_ARG(k >= 0, "multipole order must be >= 0 (got %d)", k);
    RKB_CHECK_ARG(d_fb && d_bsp && d_r && d_w && d_K, "null argument");
    const long n = (long)nv * ng;
    const size_t smem = (size_t)(2 * n + 2L * ks * ng) * sizeof(double);
    RKB_CHECK_ARG(smem <= 200 * 1024, "grid of %ld nodes too large for the exchange kernel", n);
    RKB_CUDA(set_smem(potential::exchange_column_kernel, (int)smem));
    const int threads = ns < 32 ? 32 : (ns > 1024 ? 1024 : (ns + 31) / 32 * 32);
    potential::exchange_column_kernel<<<(unsigned)ns, threads, smem, as_stream(stream)>>>(d_fb, d_bsp, d_r, d_w, nv, ng,
                                                                                         ks, ns, k, d_K);
    RKB_LAUNCHED("exchange_column_kernel");
    return RKB_OK;
}

extern "C" int rkb_occupied_density(const double *d_P, const double *d_Q, long ld, long n_orb, const double *d_occ,
                                    long target, long n, double *d_rho, void *stream) {
    RKB_CHECK_ARG(n >= 1 && ld >= n && n_orb >= 0, "invalid sizes (n=%ld, ld=%ld, n_orb=%ld)", n, ld, n_orb);
    RKB_CHECK_ARG(target < n_orb, "target orbital %ld out of range (%ld orbitals)", target, n_orb);
    RKB_CHECK_ARG(d_rho != nullptr && (n_orb == 0 || (d_P && d_Q && d_occ)), "null argument");
    potential::occupied_density_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, as_stream(stream)>>>(
        d_P, d_Q, ld, n_orb, d_occ, target, n, d_rho);
    RKB_LAUNCHED("occupied_density_kernel");
    return RKB_OK;
}

extern "C" int rkb_bspline_sym_matrix(const double *d_b1, int ks1, const double *d_b2, int ks2, int nv, int ng,
                                      const double *d_w, const double *d_f, long mm, double *d_out, void *stream) {
    RKB_CHECK_ARG(nv >= 1 && ng >= 1 && ks1 >= 1 && ks2 >= 1 && mm >= 1, "invalid sizes");
    RKB_CHECK_ARG(mm <= 1L << 15, "matrix dimension %ld too large", mm);
    RKB_CHECK_ARG(d_b1 && d_b2 && d_w && d_out, "null argument");
    const long total = mm * mm;
    potential::sym_band_matrix_kernel<<<(unsigned)ceil_div(total, 256), 256, 0, as_stream(stream)>>>(
        d_b1, ks1, d_b2, ks2, nv, ng, d_w, d_f, mm, d_out);
    RKB_LAUNCHED("sym_band_matrix_kernel");
    return RKB_OK;
}
