// Direct (Hartree) potential matrices on the device: the consumer of the Y^k
// kernel in atomx's Dirac-Fock driver (methods/dirac_fock.py:931-967,
// DFSolver._build_direct_potential_yk).
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

}  // namespace potential
}  // namespace rkb

using namespace rkb;

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
