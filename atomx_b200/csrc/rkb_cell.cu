// Cell (bank) R^k engine on the device: atomx numerics/bspline/convol.py.
//
// A bank holds the four-index integrals
//     rkb[i][j][ip][jp] = int int B_i B_{i+ip}(r1) r_<^k / r_>^(k+1) B_j B_{j+jp}(r2)
// of one component pair (P or Q basis on each electron), assembled from
// per-cell moments (cells far apart: the kernel factorises) and diagonal-cell
// integrals (nested Gauss quadrature).  Here every bank is stored as a dense
// matrix K[(ip, i)][(jp, j)] = rkb[i][j][ip][jp] (row ip*ns + i, column
// jp*ns + j) inside one block matrix per multipole,
//     K_full = [[K_pp, K_pq], [K_qp, K_qq]],
// so that with the banded pair densities of _density_sym laid out in the same
// index order, D(ab) = [D_P(ab) | D_Q(ab)], atomx's cell integral is the
// bilinear form R^k(ab, cd) = D(ab) K_full D(cd)^T.  Whole tables and batches
// of integrals are then FP64 GEMMs on the DMMA pipe plus gathered dots.
//
// The bank construction kernels keep the reference's operation order with
// explicitly rounded multiplies and adds (no fused multiply-add), so the banks
// equal atomx's bit for bit: moments (convol.py:58-94), diagonal cells
// (_triang_sym :136-250, _triang_pqpq :388-530), assembly (:324-381,
// :533-576).  So does the exchange contraction (_convol_case4_t :1001-1059)
// and the bilinear fold (_rkb_bilinear :1901-1942).
#include <cmath>

#include "rkb_common.cuh"
#include "rkb_dmma.cuh"

namespace rkb {
namespace cell {

constexpr int MAX_KS = 16;
constexpr int MAX_NSUB = 64;

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// w r^k (k > 0), w / r^-k (k < 0), w (k = 0)
__device__ __forceinline__ double power_weight(double w, double r, int k) {
    if (k > 0) return mul(w, int_pow(r, k));
    if (k < 0) return dvd(w, int_pow(r, -k));
    return w;
}

// packed upper pair (h, hp), hp >= h, of order ks: h*ks - h(h-1)/2 + (hp - h)
__device__ __forceinline__ int packed(int h, int hp, int ks) { return h * ks - (h * (h - 1)) / 2 + (hp - h); }

__device__ __forceinline__ void unpack(int p, int ks, int &h, int &hp) {
    h = 0;
    while (p >= ks - h) {
        p -= ks - h;
        ++h;
    }
    hp = h + p;
}

// B-spline values of order ks at x in the interval starting at knot `left`
// (de Boor's recurrence, the reference's _bsplvb_inplace order).
__device__ void bsplvb(const double *__restrict__ t, int ks, double x, int left, double *b) {
    double dr[MAX_KS], dl[MAX_KS];
    b[0] = 1.0;
    for (int i = 1; i < ks; ++i) b[i] = 0.0;
    for (int j = 1; j < ks; ++j) {
        dr[j] = sub(t[left + j], x);
        dl[j] = sub(x, t[left + 1 - j]);
        double saved = 0.0;
        for (int r = 0; r < j; ++r) {
            const double term = dvd(b[r], add(dr[r + 1], dl[j - r]));
            b[r] = add(saved, mul(dr[r + 1], term));
            saved = mul(dl[j - r], term);
        }
        b[j] = saved;
    }
}

// ------------------------------------------------------------------ moments
// out[ii][iv] = sum_m B_i B_j(iv, m) * power_weight(grw, gr, k), ii = packed (i, j)
__global__ void moments_kernel(const double *__restrict__ bsp, const double *__restrict__ gr,
                               const double *__restrict__ grw, int nv, int ng, int ks, int k,
                               double *__restrict__ out) {
    const int kk = ks * (ks + 1) / 2;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)kk * nv) return;
    const int ii = (int)(t / nv), iv = (int)(t % nv);
    int i, j;
    unpack(ii, ks, i, j);
    double s = 0.0;
    for (int m = 0; m < ng; ++m) {
        const double *b = bsp + ((long)iv * ng + m) * ks;
        const double gw = power_weight(grw[iv * ng + m], gr[iv * ng + m], k);
        s = add(s, mul(mul(b[i], b[j]), gw));
    }
    out[t] = s;
}

// ----------------------------------------------------------- diagonal cells
struct DiagSmem {
    double *bsub, *gwr, *span, *intp, *bw, *res_a, *res_b;
};

// One pass of the nested quadrature on cell iv: the inner integrals of the
// inner component's products (knots t_i, order ks_i) up to each outer node,
// then the outer sum with the outer component's products and the 1/r^(k+1)
// weight: res[ii_o][jj_i].
__device__ void diag_pass(const double *__restrict__ bsp_o, int ks_o, const double *__restrict__ t_i, int ks_i,
                          int iv, const double *__restrict__ gr, const double *__restrict__ grw, int ng, int k,
                          int n_sub, const double *__restrict__ x01, const double *__restrict__ w01, DiagSmem sm,
                          double *res) {
    const int left = ks_i - 1 + iv;
    const double xbase = t_i[left];
    for (int m = threadIdx.x; m < ng; m += blockDim.x) sm.span[m] = sub(gr[iv * ng + m], xbase);
    __syncthreads();
    for (int p = threadIdx.x; p < ng * n_sub; p += blockDim.x) {
        const int m = p / n_sub, n = p % n_sub;
        const double span = sm.span[m];
        double *b = sm.bsub + (long)p * ks_i;
        if (span < 1e-30) {
            for (int s = 0; s < ks_i; ++s) b[s] = 0.0;
            sm.gwr[p] = 0.0;
            continue;
        }
        const double gx = add(xbase, mul(span, x01[n]));
        bsplvb(t_i, ks_i, gx, left, b);
        const double w = mul(span, w01[n]);
        sm.gwr[p] = k > 0 ? mul(w, int_pow(gx, k)) : (k < 0 ? dvd(w, int_pow(gx, -k)) : w);
    }
    __syncthreads();
    const int kki = ks_i * (ks_i + 1) / 2, kko = ks_o * (ks_o + 1) / 2;
    for (int p = threadIdx.x; p < kki * ng; p += blockDim.x) {
        const int jj = p / ng, m = p % ng;
        int j, jp;
        unpack(jj, ks_i, j, jp);
        double s = 0.0;
        if (!(sm.span[m] < 1e-30)) {
            for (int n = 0; n < n_sub; ++n) {
                const double *b = sm.bsub + ((long)m * n_sub + n) * ks_i;
                s = add(s, mul(mul(b[j], b[jp]), sm.gwr[m * n_sub + n]));
            }
        }
        sm.intp[jj * ng + m] = s;
    }
    for (int p = threadIdx.x; p < kko * ng; p += blockDim.x) {
        const int ii = p / ng, m = p % ng;
        int i, ip;
        unpack(ii, ks_o, i, ip);
        const double ow = dvd(grw[iv * ng + m], int_pow(gr[iv * ng + m], k + 1));
        const double *bo = bsp_o + ((long)iv * ng + m) * ks_o;
        sm.bw[ii * ng + m] = mul(mul(bo[i], bo[ip]), ow);
    }
    __syncthreads();
    for (int p = threadIdx.x; p < kko * kki; p += blockDim.x) {
        const int ii = p / kki, jj = p % kki;
        double s = 0.0;
        for (int m = 0; m < ng; ++m) s = add(s, mul(sm.bw[ii * ng + m], sm.intp[jj * ng + m]));
        res[p] = s;
    }
    __syncthreads();
}

// One block per cell: out[ii_l][jj_r][iv] (kk_l x kk_r x nv).
__global__ void diag_kernel(const double *__restrict__ bsp_l, const double *__restrict__ bsp_r,
                            const double *__restrict__ gr, const double *__restrict__ grw,
                            const double *__restrict__ t_l, const double *__restrict__ t_r, int nv, int ng, int ks_l,
                            int ks_r, int same, int k, int n_sub, const double *__restrict__ x01,
                            const double *__restrict__ w01, double *__restrict__ out) {
    extern __shared__ double smem[];
    const int iv = blockIdx.x;
    const int ks_max = ks_l > ks_r ? ks_l : ks_r;
    const int kkl = ks_l * (ks_l + 1) / 2, kkr = ks_r * (ks_r + 1) / 2, kkm = ks_max * (ks_max + 1) / 2;
    DiagSmem sm;
    sm.bsub = smem;
    sm.gwr = sm.bsub + (long)ng * n_sub * ks_max;
    sm.span = sm.gwr + ng * n_sub;
    sm.intp = sm.span + ng;
    sm.bw = sm.intp + kkm * ng;
    sm.res_a = sm.bw + kkm * ng;
    sm.res_b = sm.res_a + kkl * kkr;
    // left outer, right inner: a[ii_l][jj_r]
    diag_pass(bsp_l, ks_l, t_r, ks_r, iv, gr, grw, ng, k, n_sub, x01, w01, sm, sm.res_a);
    if (same) {
        for (int p = threadIdx.x; p < kkl * kkr; p += blockDim.x) {
            const int ii = p / kkr, jj = p % kkr;
            out[(long)p * nv + iv] = add(sm.res_a[ii * kkr + jj], sm.res_a[jj * kkr + ii]);
        }
        return;
    }
    // right outer, left inner: b[jj_r][ii_l]
    diag_pass(bsp_r, ks_r, t_l, ks_l, iv, gr, grw, ng, k, n_sub, x01, w01, sm, sm.res_b);
    for (int p = threadIdx.x; p < kkl * kkr; p += blockDim.x) {
        const int ii = p / kkr, jj = p % kkr;
        out[(long)p * nv + iv] = add(sm.res_a[ii * kkr + jj], sm.res_b[jj * kkl + ii]);
    }
}

// ------------------------------------------------------------------ assembly
// One thread per bank element, stored at K[(row_off + ip*ns + i)][col_off + jp*ns + j]:
// cells iv < jv contribute rising_l[ii][iv] falling_r[jj][jv], cells iv > jv
// rising_r[jj][jv] falling_l[ii][iv], iv == jv the diagonal cell; summed over
// jv, then iv, ascending.
__global__ void assemble_kernel(const double *__restrict__ rl, const double *__restrict__ fl,
                                const double *__restrict__ rr, const double *__restrict__ fr,
                                const double *__restrict__ diag, int nv, int ks_l, int ks_r, int ns,
                                double *__restrict__ out, long ld, long row_off, long col_off) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ks_l * ns * ks_r * ns) return;
    const int j = (int)(t % ns);
    const long r1 = t / ns;
    const int jp = (int)(r1 % ks_r);
    const long r2 = r1 / ks_r;
    const int i = (int)(r2 % ns), ip = (int)(r2 / ns);
    const int kkr = ks_r * (ks_r + 1) / 2;
    const int jv_lo = max(0, j - (ks_r - 1 - jp)), jv_hi = min(j, nv - 1);
    const int iv_lo = max(0, i - (ks_l - 1 - ip)), iv_hi = min(i, nv - 1);
    double acc = 0.0;
    for (int jv = jv_lo; jv <= jv_hi; ++jv) {
        const int jh = j - jv, jj = packed(jh, jh + jp, ks_r);
        for (int iv = iv_lo; iv <= iv_hi; ++iv) {
            const int ih = i - iv, ii = packed(ih, ih + ip, ks_l);
            double c;
            if (iv < jv) c = mul(rl[(long)ii * nv + iv], fr[(long)jj * nv + jv]);
            else if (iv > jv) c = mul(rr[(long)jj * nv + jv], fl[(long)ii * nv + iv]);
            else c = diag[((long)ii * kkr + jj) * nv + iv];
            acc = add(acc, c);
        }
    }
    out[(row_off + (long)ip * ns + i) * ld + col_off + (long)jp * ns + j] = acc;
}

// ---------------------------------------------------------------- densities
// Banded pair densities of _density_sym (extent ns_d, order ks; component
// vectors of stored lengths n1, n2) in bank index order:
// out[p][col_off + s*ns_k + i] = d[i][s].
__global__ void densities_kernel(const double *__restrict__ c1, const double *__restrict__ c2, long ld,
                                 const long *__restrict__ pairs, long n_pairs, int n1, int n2, int ns_d, int ns_k,
                                 int ks, double *__restrict__ out, long out_ld, long col_off) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_pairs * ks * ns_k) return;
    const int i = (int)(t % ns_k);
    const long r = t / ns_k;
    const int s = (int)(r % ks);
    const long p = r / ks;
    const double *p1 = c1 + pairs[2 * p] * ld, *p2 = c2 + pairs[2 * p + 1] * ld;
    double v = 0.0;
    if (i < min(n1, ns_d)) {
        if (s == 0) {
            if (i < n2) v = mul(p1[i], p2[i]);
        } else {
            const int ip = i + s;
            if (ip < ns_d) {
                double x = 0.0;
                if (ip < n2) x = add(x, mul(p1[i], p2[ip]));
                if (ip < n1 && i < n2) x = add(x, mul(p1[ip], p2[i]));
                v = x;
            }
        }
    }
    out[p * out_ld + col_off + (long)s * ns_k + i] = v;
}

// ------------------------------------------------------------- FP64 GEMM NT
// C[m][n] (+)= sum_x A[m][x] B[n][x]: 128 x 128 tiles, 3-stage cp.async ring,
// mma.sync m8n8k4 f64, one persistent CTA per SM over the tile list.
constexpr int BM = 128, BN = 128, BK = 16, PAD = 4, LDS = BK + PAD, STAGES = 3, THREADS = 256;
constexpr size_t GEMM_SMEM = (size_t)STAGES * (BM + BN) * LDS * sizeof(double);

__device__ __forceinline__ void load_rows(double *s, const double *__restrict__ g, long ld, long row0, long nrows,
                                          long k0) {
#pragma unroll
    for (int it = 0; it < 4; ++it) {
        const int c = threadIdx.x + it * THREADS;
        const int row = c >> 3, col = (c & 7) * 2;
        const long grow = row0 + row;
        const bool ok = grow < nrows;
        cp_async16(s + row * LDS + col, g + (ok ? grow : row0) * ld + k0 + col, ok ? 16 : 0);
    }
}

__global__ void __launch_bounds__(THREADS, 1)
gemm_nt_kernel(const double *__restrict__ A, long lda, const double *__restrict__ B, long ldb, double *__restrict__ C,
               long ldc, long M, long N, long K, int accumulate) {
    extern __shared__ double smem[];
    double *As = smem, *Bs = smem + STAGES * BM * LDS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp >> 2, wn = warp & 3, fr = lane >> 2, fc = lane & 3;
    const long tm = (M + BM - 1) / BM, tn = (N + BN - 1) / BN;
    const int nk = (int)(K / BK);
    for (long t = blockIdx.x; t < tm * tn; t += gridDim.x) {
        const long i0 = (t / tn) * BM, j0 = (t % tn) * BN;
        double acc[8][4][2];
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
        __syncthreads();
#pragma unroll
        for (int s = 0; s < STAGES - 1; ++s) {
            if (s < nk) {
                load_rows(As + s * BM * LDS, A, lda, i0, M, (long)s * BK);
                load_rows(Bs + s * BN * LDS, B, ldb, j0, N, (long)s * BK);
            }
            cp_async_commit();
        }
        for (int kb = 0; kb < nk; ++kb) {
            cp_async_wait<STAGES - 2>();
            __syncthreads();
            const int pf = kb + STAGES - 1;
            if (pf < nk) {
                const int s = pf % STAGES;
                load_rows(As + s * BM * LDS, A, lda, i0, M, (long)pf * BK);
                load_rows(Bs + s * BN * LDS, B, ldb, j0, N, (long)pf * BK);
            }
            cp_async_commit();
            const double *a_s = As + (kb % STAGES) * BM * LDS + (wm * 64 + fr) * LDS + fc;
            const double *b_s = Bs + (kb % STAGES) * BN * LDS + (wn * 32 + fr) * LDS + fc;
#pragma unroll
            for (int kk = 0; kk < BK; kk += 4) {
                double af[8], bf[4];
#pragma unroll
                for (int a = 0; a < 8; ++a) af[a] = a_s[a * 8 * LDS + kk];
#pragma unroll
                for (int b = 0; b < 4; ++b) bf[b] = b_s[b * 8 * LDS + kk];
#pragma unroll
                for (int a = 0; a < 8; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) dmma(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
            }
        }
        cp_async_wait<0>();
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const long i = i0 + wm * 64 + a * 8 + fr;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const long j = j0 + wn * 32 + b * 8 + fc * 2;
#pragma unroll
                for (int e = 0; e < 2; ++e)
                    if (i < M && j + e < N) {
                        double *c = C + i * ldc + j + e;
                        *c = accumulate ? *c + acc[a][b][e] : acc[a][b][e];
                    }
            }
        }
    }
}

// ------------------------------------------------------------- gathered dots
// out[e] = sum_x L[il[e]][x] W[iw[e]][x], one warp per entry
__global__ void dots_kernel(const double *__restrict__ L, long l_ld, const double *__restrict__ W, long w_ld, long n,
                            const long *__restrict__ il, const long *__restrict__ iw, long n_ent,
                            double *__restrict__ out) {
    const long e = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (e >= n_ent) return;
    const double *x = L + il[e] * l_ld, *y = W + iw[e] * w_ld;
    double s = 0.0;
    for (long i = lane; i < n; i += 32) s = fma(x[i], y[i], s);
    s = warp_sum(s);
    if (lane == 0) out[e] = s;
}

// ----------------------------------------------------------------- exchange
// _convol_case4_t on one bank block: a[row][col] over the four families in
// the reference's order; `symmetric` computes col <= row and mirrors.  Bank
// element rkb[i][j][ip][jp] = K[(ip*ns + i) * ld + jp*ns + j].  Batch b uses
// density d + b*ns*ns, bank block K + kofs[b], output a + b*ns*ns.
__global__ void exchange_kernel(const double *__restrict__ K, long ld, const long *__restrict__ kofs,
                                const double *__restrict__ d, int ns, int ks, int ks_r, int symmetric,
                                int accumulate, double *__restrict__ a, long nbatch) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long per = (long)ns * ns;
    if (t >= per * nbatch) return;
    const long b = t / per;
    const int row = (int)((t % per) / ns), col = (int)(t % ns);
    if (symmetric && col > row) return;
    const double *Kb = K + kofs[b];
    const double *db = d + b * per;
#define RKB(i, j, ip, jp) Kb[((long)(ip) * ns + (i)) * ld + (long)(jp) * ns + (j)]
    double s = 0.0;
    for (int ip = 0; ip < ks; ++ip) {
        const int i = row - ip;
        if (i < 0) continue;
        for (int jp = 0; jp < ks_r; ++jp)
            if (col < ns - jp) s = add(s, mul(RKB(i, col, ip, jp), db[(long)i * ns + col + jp]));
    }
    for (int ip = 1; ip < ks; ++ip) {
        const int ii = row + ip;
        if (ii >= ns) continue;
        for (int jp = 0; jp < ks_r; ++jp)
            if (col < ns - jp) s = add(s, mul(RKB(row, col, ip, jp), db[(long)ii * ns + col + jp]));
    }
    for (int jp = 1; jp < ks_r; ++jp)
        for (int ip = 0; ip < ks; ++ip) {
            const int i = row - ip;
            if (i < 0) continue;
            if (col >= jp) s = add(s, mul(RKB(i, col - jp, ip, jp), db[(long)i * ns + col - jp]));
        }
    for (int ip = 1; ip < ks; ++ip) {
        const int ii = row + ip;
        if (ii >= ns) continue;
        for (int jp = 1; jp < ks_r; ++jp)
            if (col >= jp) s = add(s, mul(RKB(row, col - jp, ip, jp), db[(long)ii * ns + col - jp]));
    }
#undef RKB
    double *o = a + b * per + (long)row * ns + col;
    *o = accumulate ? add(*o, s) : s;
    if (symmetric && col < row) {
        double *m = a + b * per + (long)col * ns + row;
        *m = accumulate ? add(*m, s) : s;
    }
}

// ----------------------------------------------------------------- bilinear
// _rkb_bilinear stage 1, gathered: T[m][j][jp] over the reference's scatter
// order (left pairs i = m - ip for ip = ks_l-1..1, then i = m with ip = 0..).
__global__ void bilinear_t_kernel(const double *__restrict__ K, long ld, int ns, const double *__restrict__ wa,
                                  int n_left, int n_right, int ks_l, int ks_r, int ns_out, double *__restrict__ T) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ns_out * n_right * ks_r) return;
    const int jp = (int)(t % ks_r);
    const long r = t / ks_r;
    const int j = (int)(r % n_right), m = (int)(r / n_right);
#define RKB(i, j, ip, jp) K[((long)(ip) * ns + (i)) * ld + (long)(jp) * ns + (j)]
    double s = 0.0;
    if (j + jp < n_right) {
        for (int i = max(0, m - (ks_l - 1)); i < m; ++i) {  // i + ip = m, ip = m - i > 0
            if (i >= n_left || m >= n_left) continue;
            s = add(s, mul(RKB(i, j, m - i, jp), wa[i]));
        }
        if (m < n_left)
            for (int ip = 0; ip < ks_l; ++ip) {
                if (m + ip >= n_left) break;
                s = add(s, mul(RKB(m, j, ip, jp), wa[m + ip]));
            }
    }
#undef RKB
    T[t] = s;
}

// stage 2: M[m][n] from T over the reference's order (right pairs j = n - jp
// for jp = ks_r-1..1, then j = n with jp = 0..)
__global__ void bilinear_m_kernel(const double *__restrict__ T, const double *__restrict__ wb, int n_right, int ks_r,
                                  int ns_out, double *__restrict__ M) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ns_out * ns_out) return;
    const int n = (int)(t % ns_out), m = (int)(t / ns_out);
    const double *Tm = T + (long)m * n_right * ks_r;
    double s = 0.0;
    for (int j = max(0, n - (ks_r - 1)); j < n; ++j) {  // j + jp = n, jp > 0
        if (j >= n_right || n >= n_right) continue;
        s = add(s, mul(Tm[(long)j * ks_r + (n - j)], wb[j]));
    }
    if (n < n_right)
        for (int jp = 0; jp < ks_r; ++jp) {
            if (n + jp >= n_right) break;
            s = add(s, mul(Tm[(long)n * ks_r + jp], wb[n + jp]));
        }
    M[t] = s;
}

// ------------------------------------------------------- Fock-block helpers
// Direct density of one (target, block, k): dd[s*ns + i] = sum_j c_j (doubled
// for j = target) of the symmetric band of comp[j] (convol.py:647-686).
__global__ void direct_density_kernel(const double *__restrict__ comp, long ld, int n_orb,
                                      const double *__restrict__ coef, long coef_stride, const int *__restrict__ target,
                                      int ns, int ks, double *__restrict__ dd, long out_ld, long nbatch) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ns * ks * nbatch) return;
    const long b = t / ((long)ns * ks);
    const int s = (int)((t / ns) % ks), i = (int)(t % ns);
    const double *c = coef + b * coef_stride;
    double v = 0.0;
    if (i + s < ns)
        for (int j = 0; j < n_orb; ++j) {
            double cj = c[j];
            if (cj == 0.0) continue;
            if (j == target[b]) cj = add(cj, cj);
            const double pi = comp[(long)j * ld + i];
            if (s == 0) v = add(v, mul(mul(cj, pi), pi));
            else {
                const double ps = comp[(long)j * ld + i + s];
                v = add(v, mul(cj, add(mul(pi, ps), mul(ps, pi))));
            }
        }
    dd[b * out_ld + (long)s * ns + i] = v;
}

// Exchange density: xx[i][k] = sum_j (c_j comp_ii[j][i]) comp_jj[j][k] (convol.py:689-710)
__global__ void exchange_density_kernel(const double *__restrict__ comp_ii, const double *__restrict__ comp_jj,
                                        long ld, int n_orb, const double *__restrict__ coef, long coef_stride, int ns,
                                        double *__restrict__ xx, long nbatch) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long per = (long)ns * ns;
    if (t >= per * nbatch) return;
    const long b = t / per;
    const int i = (int)((t % per) / ns), kk = (int)(t % ns);
    const double *c = coef + b * coef_stride;
    double v = 0.0;
    for (int j = 0; j < n_orb; ++j) {
        const double cj = c[j];
        if (cj == 0.0) continue;
        v = add(v, mul(mul(cj, comp_ii[(long)j * ld + i]), comp_jj[(long)j * ld + kk]));
    }
    xx[t] = v;
}

// Banded potential to a full symmetric matrix: V[i][i+s] += v[s*ns + i] and
// its mirror (convol.py:815-826).  One thread per (i, s); rows of one batch
// element touch disjoint entries for distinct (i, s).
__global__ void banded_to_full_kernel(const double *__restrict__ v, int ns, int ks, double *__restrict__ V,
                                      long nbatch) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ns * ks * nbatch) return;
    const long b = t / ((long)ns * ks);
    const int s = (int)((t / ns) % ks), i = (int)(t % ns);
    if (i + s >= ns) return;
    const double val = v[t];
    double *Vb = V + b * (long)ns * ns;
    Vb[(long)i * ns + i + s] = add(Vb[(long)i * ns + i + s], val);
    if (s > 0) Vb[(long)(i + s) * ns + i] = add(Vb[(long)(i + s) * ns + i], val);
}

// Fock blocks: PP = 0.5 (PP + PP^T), QQ likewise, PQ = 0.5 (PQ + QP^T) (or
// QP^T when the PQ exchange was skipped), QP = PQ^T, all divided by the norm
// when it exceeds 1e-15 (dirac_fock.py:1295-1319).  h holds PP, QQ, PQ, QP of
// each batch element (4 ns x ns); out receives the result.
__global__ void fock_finish_kernel(const double *__restrict__ h, const double *__restrict__ norm, int ns,
                                   int skip_pq, double *__restrict__ out, long nbatch) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long per = (long)ns * ns;
    if (t >= per * nbatch) return;
    const long b = t / per;
    const int i = (int)((t % per) / ns), j = (int)(t % ns);
    const double *H = h + b * 4 * per;
    double *O = out + b * 4 * per;
    const double nb = norm[b];
    auto fin = [&](double x) { return nb > 1e-15 ? x / nb : x; };
    const long ij = (long)i * ns + j, ji = (long)j * ns + i;
    O[ij] = fin(0.5 * (H[ij] + H[ji]));
    O[per + ij] = fin(0.5 * (H[per + ij] + H[per + ji]));
    const double pq = skip_pq ? H[3 * per + ji] : 0.5 * (H[2 * per + ij] + H[3 * per + ji]);
    const double qp = skip_pq ? H[3 * per + ij] : 0.5 * (H[2 * per + ji] + H[3 * per + ij]);
    O[2 * per + ij] = fin(pq);
    O[3 * per + ij] = fin(qp);
}

}  // namespace cell
}  // namespace rkb

using namespace rkb;

// ----------------------------------------------------------------- host side
namespace {
inline unsigned blocks_for(long n, int threads = 256) { return (unsigned)ceil_div(n, threads); }
}

extern "C" void rkb_gauss_legendre_01(int n, double *x, double *w) {
    if (n == 1) {
        x[0] = 0.5;
        w[0] = 1.0;
        return;
    }
    // Newton's iteration on the Legendre three-term recurrence from the
    // Chebyshev-like guess cos(pi (i + 3/4) / (n + 1/2)), then mapped to [0, 1]
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < n; ++i) {
        double xi = std::cos(pi * (i + 0.75) / (n + 0.5)), p0 = 1.0, p1 = xi, dp = 0.0;
        for (int it = 0; it < 50; ++it) {
            p0 = 1.0;
            p1 = xi;
            for (int j = 2; j <= n; ++j) {
                const double p2 = ((2 * j - 1) * xi * p1 - (j - 1) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (xi * p1 - p0) / (xi * xi - 1.0);
            const double dx = p1 / dp;
            xi -= dx;
            if (std::fabs(dx) < 1e-15) break;
        }
        x[i] = 0.5 * (xi + 1.0);
        w[i] = 1.0 / ((1.0 - xi * xi) * dp * dp);
    }
}

extern "C" int rkb_cell_moments(const double *d_bsp, const double *d_gr, const double *d_grw, int nv, int ng, int ks,
                                int k, double *d_out, void *stream) {
    RKB_CHECK_ARG(nv >= 1 && ng >= 1 && ng <= RKB_MAX_NG && ks >= 1 && ks <= cell::MAX_KS, "invalid basis sizes");
    RKB_CHECK_ARG(k >= -64 && k <= 64, "multipole power out of range (%d)", k);
    const long n = (long)ks * (ks + 1) / 2 * nv;
    cell::moments_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(d_bsp, d_gr, d_grw, nv, ng, ks, k, d_out);
    RKB_LAUNCHED("cell::moments_kernel");
    return RKB_OK;
}

static size_t diag_smem(int ng, int n_sub, int ks_l, int ks_r) {
    const int ksm = ks_l > ks_r ? ks_l : ks_r;
    const long kkl = ks_l * (ks_l + 1) / 2, kkr = ks_r * (ks_r + 1) / 2, kkm = ksm * (ksm + 1) / 2;
    return sizeof(double) * ((size_t)ng * n_sub * ksm + (size_t)ng * n_sub + ng + 2 * kkm * ng + 2 * kkl * kkr);
}

extern "C" int rkb_cell_diag(const double *d_bsp_l, const double *d_bsp_r, const double *d_gr, const double *d_grw,
                             const double *d_t_l, const double *d_t_r, int nv, int ng, int ks_l, int ks_r, int same,
                             int k, const double *d_x01, const double *d_w01, int n_sub, double *d_out, void *stream) {
    RKB_CHECK_ARG(nv >= 1 && ng >= 1 && ng <= RKB_MAX_NG, "invalid grid");
    RKB_CHECK_ARG(ks_l >= 1 && ks_l <= cell::MAX_KS && ks_r >= 1 && ks_r <= cell::MAX_KS, "orders must be 1..%d",
                  cell::MAX_KS);
    RKB_CHECK_ARG(n_sub >= 1 && n_sub <= cell::MAX_NSUB, "sub-quadrature order must be 1..%d", cell::MAX_NSUB);
    RKB_CHECK_ARG(k >= 0 && k <= 64, "multipole rank must be in [0, 64] (got %d)", k);
    RKB_CHECK_ARG(!same || ks_l == ks_r, "a same-component cell needs equal orders");
    const size_t smem = diag_smem(ng, n_sub, ks_l, ks_r);
    RKB_CHECK_ARG(smem <= 200 * 1024, "diagonal-cell workspace too large (%zu bytes)", smem);
    RKB_CUDA(set_smem(cell::diag_kernel, (int)smem));
    cell::diag_kernel<<<(unsigned)nv, 256, smem, as_stream(stream)>>>(d_bsp_l, d_bsp_r, d_gr, d_grw, d_t_l, d_t_r, nv,
                                                                       ng, ks_l, ks_r, same, k, n_sub, d_x01, d_w01,
                                                                       d_out);
    RKB_LAUNCHED("cell::diag_kernel");
    return RKB_OK;
}

extern "C" int rkb_cell_assemble(const double *d_rising_l, const double *d_falling_l, const double *d_rising_r,
                                 const double *d_falling_r, const double *d_diag, int nv, int ks_l, int ks_r, int ns,
                                 double *d_out, long ld, long row_off, long col_off, void *stream) {
    RKB_CHECK_ARG(nv >= 1 && ns >= 1 && ks_l >= 1 && ks_l <= cell::MAX_KS && ks_r >= 1 && ks_r <= cell::MAX_KS,
                  "invalid bank sizes");
    RKB_CHECK_ARG(row_off >= 0 && col_off >= 0 && ld >= col_off + (long)ks_r * ns, "bank block outside the matrix");
    const long n = (long)ks_l * ns * ks_r * ns;
    cell::assemble_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(d_rising_l, d_falling_l, d_rising_r,
                                                                        d_falling_r, d_diag, nv, ks_l, ks_r, ns, d_out,
                                                                        ld, row_off, col_off);
    RKB_LAUNCHED("cell::assemble_kernel");
    return RKB_OK;
}

extern "C" int rkb_cell_densities(const double *d_c1, const double *d_c2, long ld, const long *d_pairs, long n_pairs,
                                  int n1, int n2, int ns_d, int ns_k, int ks, double *d_out, long out_ld, long col_off,
                                  void *stream) {
    RKB_CHECK_ARG(n1 >= 0 && n2 >= 0 && n1 <= ld && n2 <= ld && ns_d >= 1 && ns_d <= ns_k && ks >= 1,
                  "invalid density sizes");
    RKB_CHECK_ARG(col_off >= 0 && out_ld >= col_off + (long)ks * ns_k, "density block outside the row");
    if (n_pairs == 0) return RKB_OK;
    const long n = n_pairs * ks * ns_k;
    cell::densities_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(d_c1, d_c2, ld, d_pairs, n_pairs, n1, n2,
                                                                         ns_d, ns_k, ks, d_out, out_ld, col_off);
    RKB_LAUNCHED("cell::densities_kernel");
    return RKB_OK;
}

extern "C" int rkb_gemm_nt_fp64(const double *d_A, long lda, const double *d_B, long ldb, double *d_C, long ldc,
                                long M, long N, long K, int accumulate, void *stream) {
    RKB_CHECK_ARG(M >= 0 && N >= 0 && K >= 0 && K % cell::BK == 0, "K (%ld) must be a multiple of %d", K, cell::BK);
    RKB_CHECK_ARG(lda >= K && ldb >= K && ldc >= N && lda % 2 == 0 && ldb % 2 == 0,
                  "leading dimensions must cover the matrices (and lda, ldb be even)");
    RKB_CHECK_ARG(((uintptr_t)d_A % 16) == 0 && ((uintptr_t)d_B % 16) == 0, "A and B must be 16-byte aligned");
    if (M == 0 || N == 0) return RKB_OK;
    const long tiles = ceil_div(M, cell::BM) * ceil_div(N, cell::BN);
    const long grid = tiles < sm_count() ? tiles : sm_count();
    RKB_CUDA(set_smem(cell::gemm_nt_kernel, (int)cell::GEMM_SMEM));
    cell::gemm_nt_kernel<<<(unsigned)grid, cell::THREADS, cell::GEMM_SMEM, as_stream(stream)>>>(
        d_A, lda, d_B, ldb, d_C, ldc, M, N, K, accumulate);
    RKB_LAUNCHED("cell::gemm_nt_kernel");
    return RKB_OK;
}

extern "C" int rkb_cell_dots(const double *d_L, long l_ld, const double *d_W, long w_ld, long n, const long *d_il,
                             const long *d_iw, long n_ent, double *d_out, void *stream) {
    RKB_CHECK_ARG(n >= 0 && l_ld >= n && w_ld >= n, "invalid sizes");
    if (n_ent == 0) return RKB_OK;
    cell::dots_kernel<<<(unsigned)ceil_div(n_ent, 8), 256, 0, as_stream(stream)>>>(d_L, l_ld, d_W, w_ld, n, d_il,
                                                                                  d_iw, n_ent, d_out);
    RKB_LAUNCHED("cell::dots_kernel");
    return RKB_OK;
}

extern "C" int rkb_cell_exchange(const double *d_K, long ld, const long *d_kofs, const double *d_dens, long nbatch,
                                 int ns, int ks_l, int ks_r, int symmetric, int accumulate, double *d_out,
                                 void *stream) {
    RKB_CHECK_ARG(ns >= 1 && ks_l >= 1 && ks_r >= 1 && ld >= (long)ks_r * ns, "invalid sizes");
    RKB_CHECK_ARG(!symmetric || ks_l == ks_r, "a symmetric exchange needs equal orders");
    if (nbatch == 0) return RKB_OK;
    const long n = (long)ns * ns * nbatch;
    cell::exchange_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(d_K, ld, d_kofs, d_dens, ns, ks_l, ks_r,
                                                                        symmetric, accumulate, d_out, nbatch);
    RKB_LAUNCHED("cell::exchange_kernel");
    return RKB_OK;
}

extern "C" int rkb_cell_bilinear(const double *d_K, long ld, int ns, const double *d_wa, const double *d_wb,
                                 int n_left, int n_right, int ks_l, int ks_r, int ns_out, double *d_T, double *d_M,
                                 void *stream) {
    RKB_CHECK_ARG(ns >= 1 && n_left >= 0 && n_left <= ns && n_right >= 0 && n_right <= ns && ns_out >= n_left &&
                      ns_out >= n_right && ld >= (long)ks_r * ns,
                  "invalid bilinear sizes");
    const long nt = (long)ns_out * n_right * ks_r, nm = (long)ns_out * ns_out;
    if (nt > 0) {
        cell::bilinear_t_kernel<<<blocks_for(nt), 256, 0, as_stream(stream)>>>(d_K, ld, ns, d_wa, n_left, n_right,
                                                                               ks_l, ks_r, ns_out, d_T);
        RKB_LAUNCHED("cell::bilinear_t_kernel");
    }
    if (nm > 0) {
        cell::bilinear_m_kernel<<<blocks_for(nm), 256, 0, as_stream(stream)>>>(d_T, d_wb, n_right, ks_r, ns_out, d_M);
        RKB_LAUNCHED("cell::bilinear_m_kernel");
    }
    return RKB_OK;
}

extern "C" int rkb_cell_direct_density(const double *d_comp, long ld, int n_orb, const double *d_coef,
                                       long coef_stride, const int *d_target, long nbatch, int ns, int ks,
                                       double *d_out, long out_ld, void *stream) {
    RKB_CHECK_ARG(ns >= 1 && ks >= 1 && ld >= ns && n_orb >= 0 && out_ld >= (long)ks * ns, "invalid sizes");
    if (nbatch == 0) return RKB_OK;
    const long n = (long)ns * ks * nbatch;
    cell::direct_density_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(d_comp, ld, n_orb, d_coef, coef_stride,
                                                                              d_target, ns, ks, d_out, out_ld, nbatch);
    RKB_LAUNCHED("cell::direct_density_kernel");
    return RKB_OK;
}

extern "C" int rkb_cell_exchange_density(const double *d_comp_ii, const double *d_comp_jj, long ld, int n_orb,
                                         const double *d_coef, long coef_stride, long nbatch, int ns, double *d_out,
                                         void *stream) {
    RKB_CHECK_ARG(ns >= 1 && ld >= ns && n_orb >= 0, "invalid sizes");
    if (nbatch == 0) return RKB_OK;
    const long n = (long)ns * ns * nbatch;
    cell::exchange_density_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(d_comp_ii, d_comp_jj, ld, n_orb,
                                                                                d_coef, coef_stride, ns, d_out,
                                                                                nbatch);
    RKB_LAUNCHED("cell::exchange_density_kernel");
    return RKB_OK;
}

extern "C" int rkb_cell_banded_to_full(const double *d_v, int ns, int ks, long nbatch, double *d_V, void *stream) {
    RKB_CHECK_ARG(ns >= 1 && ks >= 1, "invalid sizes");
    if (nbatch == 0) return RKB_OK;
    const long n = (long)ns * ks * nbatch;
    cell::banded_to_full_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(d_v, ns, ks, d_V, nbatch);
    RKB_LAUNCHED("cell::banded_to_full_kernel");
    return RKB_OK;
}

extern "C" int rkb_cell_fock_finish(const double *d_h, const double *d_norm, int ns, int skip_pq, long nbatch,
                                    double *d_out, void *stream) {
    RKB_CHECK_ARG(ns >= 1 && d_h != d_out, "invalid sizes (the output must not alias the input)");
    if (nbatch == 0) return RKB_OK;
    const long n = (long)ns * ns * nbatch;
    cell::fock_finish_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(d_h, d_norm, ns, skip_pq, d_out, nbatch);
    RKB_LAUNCHED("cell::fock_finish_kernel");
    return RKB_OK;
}
