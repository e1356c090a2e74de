/*
 * rkb200 — B200-native engine for relativistic radial Slater integrals R^k.
 *
 * C-ABI boundary.  Every pointer argument named d_* is a DEVICE pointer on the
 * calling thread's current CUDA device; `stream` is a cudaStream_t passed as
 * void* (NULL = legacy default stream).  Arrays are C-order float64 unless a
 * type says otherwise.  Every entry point is asynchronous with respect to the
 * host unless stated, returns an rkb_status, and never allocates device memory
 * except where its comment says so.
 *
 * Each entry point names the reference interface (atomx, path relative to
 * its project root) whose arguments and meaning it mirrors.
 */
#ifndef RKB200_H
#define RKB200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    RKB_OK = 0,
    RKB_EINVAL = 1,        /* bad size, stride, multipole or method (reference: ValueError) */
    RKB_ENONFINITE = 2,    /* non-finite value in a result (reference: FloatingPointError) */
    RKB_ENOMEM = 3,        /* workspace or admission limit exceeded (reference: MemoryError) */
    RKB_ETIMEDOUT = 4,     /* a bounded device-side wait gave up */
    RKB_ECUDA = 5,         /* CUDA runtime error; see rkb_last_error() */
    RKB_EUNSUPPORTED = 6   /* device is not sm_100 or feature not built */
} rkb_status;

/* Text of the last error raised on this host thread (never NULL). */
const char *rkb_last_error(void);

/* Library version string and compiled device architecture. */
const char *rkb_version(void);

/* 1 if the current device can run the kernels of this library (sm_100), else 0. */
int rkb_device_supported(void);

/* Largest Gauss order per cell accepted by the Y^k kernels. */
#define RKB_MAX_NG 32

/* ---------------------------------------------------------------------------
 * Y^k on the dense Gauss grid.
 *
 * rkb_yk_flat mirrors atomx numerics/yk.py:88 yk_flat(rho_flat, r_flat,
 * w_flat, n, k, nv, ng, mo, mi) -> yk (n,): outward cell sums with the
 * interpolatory partial matrix mo, inward with mi, Y = r^-(k+1) I_out + r^k I_in.
 * d_mo, d_mi are ng x ng row-major (atomx yk_partial_matrices).
 * ------------------------------------------------------------------------- */
int rkb_yk_flat(const double *d_rho, const double *d_r, const double *d_w, long n, int k,
                int nv, int ng, const double *d_mo, const double *d_mi, double *d_yk,
                void *stream);

/* Batched rows: row q reads density d_rho + q*rho_ld, uses multipole
 * d_row_k[q] and writes d_yk + q*yk_ld.  Same rule as rkb_yk_flat
 * (atomx numerics/yk.py:157 compute_yk applied per row).  In both, the
 * output must not overlap the density (RKB_EINVAL): the output rows hold
 * the outward sums until the inward pass has read the density again. */
int rkb_yk_rows(const double *d_rho, long rho_ld, const int *d_row_k, long nrows,
                const double *d_r, const double *d_w, int nv, int ng,
                const double *d_mo, const double *d_mi, double *d_yk, long yk_ld,
                void *stream);

/* ---------------------------------------------------------------------------
 * Orbital values on the grid: out[o, iv*ng+m] = sum_s coeff[o, iv+s] * bsp[iv, m, s],
 * with coefficients at index >= ns taken as zero.
 * Mirrors atomx numerics/bspline/evaluate.py:71 eval_orbital_on_grid(coeffs,
 * bsp, nv, ks, ns), batched over n_orb coefficient rows.
 * ------------------------------------------------------------------------- */
int rkb_eval_orbitals(const double *d_coeff, long coeff_ld, long n_orb, const double *d_bsp,
                      int nv, int ng, int ks, int ns, double *d_out, long out_ld, void *stream);

/* Dirac pair densities rho[p] = P[a]P[c] + Q[a]Q[c] for pairs d_pairs[2p], d_pairs[2p+1]
 * (atomx numerics/bspline/slater_yk.py:193-194). */
int rkb_pair_density(const double *d_P, const double *d_Q, long orb_ld, const long *d_pairs,
                     long n_pairs, long n, double *d_rho, long rho_ld, void *stream);

/* The upper triangle (j >= i) of a symmetric n x n row-major table, packed
 * row by row: packed[i*n - i(i-1)/2 + (j - i)] = T[i][j], n(n+1)/2 doubles.
 * Every ordered entry of an R^k table, R^k(ac;bd) = R^k(bd;ac), is in it;
 * the engine ships tables to the host in this form (atomx returns each
 * integral separately, numerics/bspline/slater.py:118). */
int rkb_pack_upper(const double *d_table, long n, double *d_packed, void *stream);

/* Quadrature dots out[e] = sum_i w_i a[ia[e]]_i b[ib[e]]_i (atomx
 * numerics/bspline/slater.py:130, the slater_rk_poisson contraction). */
int rkb_weighted_dots(const double *d_a, long a_ld, const double *d_b, long b_ld,
                      const double *d_w, long n, const long *d_ia, const long *d_ib,
                      long n_ent, double *d_out, void *stream);

/* O(N^2) direct integrator with the coincident cell split along r = s
 * (atomx numerics/bspline/slater.py:81 slater_rk_direct).  d_rho13 / d_rho24
 * are (nv*ng); xi0 is the first node of the ng-point Gauss rule on [-1, 1];
 * d_outer (order x ng), d_inner (order*order x ng), d_x, d_wx (order) describe
 * the triangle rule; d_out receives one double. */
int rkb_slater_direct(const double *d_rho13, const double *d_rho24, const double *d_r,
                      const double *d_w, int nv, int ng, int k, int order, double xi0,
                      const double *d_x, const double *d_wx, const double *d_outer,
                      const double *d_inner, double *d_out, void *stream);

/* ---------------------------------------------------------------------------
 * Arbitrary-grid trapezoid Y^k (atomx numerics/quadrature.py).
 *
 * Tables for a grid r[n] and ranks 0..K (atomx quadrature.py:190-231
 * _coulomb_tables): d_RK and d_inverse are (K+1) x n (block-scaled r^k and
 * r^-(k+1)), d_cuts[ncuts] the frame starts (d_cuts[ncuts-1] = n) and
 * d_transfers (K+1) x ntr (ntr >= ncuts-2) the frame-change factors.
 *
 * rkb_grid_yk_rows mirrors quadrature.py:234 yk_on_grid per row: row m
 * reads d_rho + m*rho_ld and rank d_rows_k[m], and writes Y^k at points
 * 0..i_cut of d_y + m*y_ld.
 *
 * rkb_grid_pair_dot_batch mirrors quadrature.py:282 yk_pair_dot_batch_on_grid:
 * row m forms rho = PA[a]PB[b] + QA[a]QB[b] (a = d_rows_a[m], b =
 * d_rows_b[m], rows of stride ld), takes Y^k (k = d_rows_k[m]) on points
 * 0..i_cut and, for each consumer slot s in [d_cons_ptr[m], d_cons_ptr[m+1]),
 * writes d_val[s] = sum_i W[d_cons_rho[s]][i] Y_i (W rows of stride w_ld).
 * Rows with d_rows_ok[m] == 0 leave their slots untouched (zero them first).
 * d_work: work_rows x n doubles of scratch (one row per concurrent CTA).
 * ------------------------------------------------------------------------- */
int rkb_grid_yk_rows(const double *d_rho, long rho_ld, const long *d_rows_k, long nrows,
                     const double *d_r, long n, const double *d_RK, const double *d_inverse,
                     const long *d_cuts, long ncuts, const double *d_transfers, long ntr, long i_cut,
                     double *d_y, long y_ld, void *stream);

int rkb_grid_pair_dot_batch(const double *d_PA, const double *d_QA, const double *d_PB,
                            const double *d_QB, long ld, const long *d_rows_a, const long *d_rows_b,
                            const long *d_rows_k, const unsigned char *d_rows_ok, long nrows,
                            const double *d_W, long w_ld, const long *d_cons_ptr,
                            const long *d_cons_rho, const double *d_r, long n, const double *d_RK,
                            const double *d_inverse, const long *d_cuts, long ncuts,
                            const double *d_transfers, long ntr, long i_cut, double *d_val,
                            double *d_work, long work_rows, void *stream);

/* ---------------------------------------------------------------------------
 * Plain FP64 table engine (all arithmetic in FP64).
 *
 * rkb_table_rows_fp64: for each row q of a plan (pair d_row_pair[q], multipole
 * d_row_k[q]) form rho from the orbital values, write g_q = w*rho into
 * d_g + q*ld and Y^k[rho] into d_y + q*ld, padding columns n..ld-1 with 0.
 *
 * rkb_table_contract_fp64: for each task t (d_tasks[3t..3t+2] = group, tile_i,
 * tile_j with tile_j >= tile_i, 128 x 128 tiles) of a group (a multipole)
 * with rows [d_grp_row0[g], +d_grp_n[g]) computes
 *     R_g[i][j] = sum_x d_g[row0+i][x] * d_y[row0+j][x]
 * into the n x n row-major block at d_out + d_grp_out[g]; tiles above the
 * diagonal are also written transposed, so the block holds every ordered
 * entry (the table of atomx slater_rk_poisson values over the group's pairs).
 * ------------------------------------------------------------------------- */
int rkb_table_rows_fp64(const double *d_Pv, const double *d_Qv, long orb_ld, const long *d_pairs,
                        const long *d_row_pair, const int *d_row_k, long nrows,
                        const double *d_r, const double *d_w, int nv, int ng,
                        const double *d_mo, const double *d_mi, double *d_g, double *d_y,
                        long ld, void *stream);

int rkb_table_contract_fp64(const double *d_g, const double *d_y, long ld, long kdim,
                            const long *d_grp_row0, const long *d_grp_n, const long *d_grp_out,
                            const int *d_tasks, long n_tasks, double *d_out, void *stream);

/* As rkb_table_contract_fp64 with a contraction length per group,
 * d_grp_kdim[g] (each a multiple of 16 and <= max_kdim <= ld): one
 * persistent launch over the groups of many ions with different grids, whose
 * rows share one (g, y) matrix of stride ld (atomx has no batched
 * counterpart; each group is a table of slater_rk_poisson values). */
int rkb_table_contract_fp64_groups(const double *d_g, const double *d_y, long ld, long max_kdim,
                                   const long *d_grp_kdim, const long *d_grp_row0, const long *d_grp_n,
                                   const long *d_grp_out, const int *d_tasks, long n_tasks,
                                   double *d_out, void *stream);

/* ---------------------------------------------------------------------------
 * Direct (Hartree) potential of the Dirac-Fock driver, the consumer of Y^0:
 * atomx methods/dirac_fock.py:931-967 (DFSolver._build_direct_potential_yk)
 * with numerics/bspline/integrals.py:18-56 (_assemble_integral).
 *
 * rkb_occupied_density: rho[i] = sum_o occ[o] (P[o][i]^2 + Q[o][i]^2), minus
 * P[target][i]^2 + Q[target][i]^2 when target >= 0; orbital values are rows
 * of leading dimension ld (n nodes); accumulated orbital by orbital in the
 * reference's order.  d_occ is a device array of n_orb doubles.
 *
 * rkb_bspline_sym_matrix: the mm x mm matrix 0.5 (M + M^T) with
 * M[gi][gj] = sum over cells iv of sum_m w[iv][m] f[iv][m] B1[iv][m][gi-iv]
 * B2[iv][m][gj-iv] (0 <= gi-iv < ks1, 0 <= gj-iv < ks2; f may be NULL for 1),
 * B1/B2 of shape (nv, ng, ks1/ks2); zero off the band.
 * ------------------------------------------------------------------------- */
int rkb_occupied_density(const double *d_P, const double *d_Q, long ld, long n_orb, const double *d_occ,
                         long target, long n, double *d_rho, void *stream);
int rkb_bspline_sym_matrix(const double *d_b1, int ks1, const double *d_b2, int ks2, int nv, int ng,
                           const double *d_w, const double *d_f, long mm, double *d_out, void *stream);

/* rkb_exchange_matrix: the ns x ns non-local exchange matrix of atomx
 * numerics/bspline/slater_yk.py:34-122 (_exchange_matrix_kernel, called by
 * compute_exchange_matrix :125):
 *     K[m][n] = sum_i w_i fb_i B_m(r_i) Y^k[fb B_n](r_i),
 * Y^k from rectangle-rule cumulative sums (not the interpolatory rule of
 * rkb_yk_rows): Y_i = r_i^-(k+1) sum_{j<=i} w_j rho_j r_j^k
 *                   + r_i^k sum_{j>=i} w_j rho_j r_j^-(k+1).
 * fb (nv*ng) is the orbital on the grid, bsp (nv, ng, ks) the B-spline
 * values, r/w the flat grid, ns <= nv + ks - 1.  Every sum runs in the
 * reference's order. */
int rkb_exchange_matrix(const double *d_fb, const double *d_bsp, const double *d_r, const double *d_w, int nv,
                        int ng, int ks, int ns, int k, double *d_K, void *stream);

/* ---------------------------------------------------------------------------
 * Split-precision engine (factored Green operator + CRT INT8 GEMMs).
 *
 * With g = w*rho, atomx's R^k(ac;bd) = g_ac^T G g_bd (numerics/yk.py:88 and
 * numerics/bspline/slater.py:130).  The engine writes
 *     R = X_ac.X_bd - Z_ac.Z_bd + left_ac.right_bd
 * with X, Z from a block Cholesky of the body of G (cells >= 1), and
 * left/right the FP64 terms of the core cell 0 and its rank-one coupling to
 * the body: left = [g_0, alpha sx, q/sx, 0...], right = [G_00 g_0, q/sx,
 * alpha sx, 0...] with alpha = v_0.g_0, q = u_b.g_b and the per-(grid, k)
 * scale sx of the factor table.
 *
 * rkb_split_rows: per plan row q (pair d_row_pair[q], multipole d_row_k[q])
 * compute [X | Z], scale by 2^(bits - e_q) so |x| < 2^bits, round, and write
 * int8 residues x mod moduli[i] to d_resA[i][row_base+q][0..kpad) (d_resB, if
 * not NULL, gets the same with Z negated), 2^(e_q - bits) to d_rowscale, the
 * core vectors (width cwp >= ng + 2) to d_left / d_right, and the row record
 * d_cbound[8q .. 8q+7]: |g_0|, |G_00 g_0|, |alpha sx|, |q/sx| divided by 2^e_q
 * (>= the row maximum of |[X | Z]|; the contraction's correction screen),
 * |[X | Z]| and the FP64 diagonal R_qq = |X|^2 - |Z|^2 + left.right (the
 * certificate's inputs), 0, 0.  d_ktab holds the per-k factor tables at
 * offsets d_koff[k] (layout at rkb_green_factor) and d_zcount[k] their
 * Z-column counts.  d_xwork is caller-provided scratch of (row_base + nrows)
 * x kpad doubles that receives the FP64 rows [X | Z | 0] before they are
 * rounded.  A row with a non-finite value gets a NaN scale and zero residues,
 * so every entry it reaches comes out NaN.
 * `moduli` is a HOST array of n_mod pairwise-coprime ints <= 256.
 *
 * rkb_split_contract: for every task (group, tile_i, tile_j >= tile_i) the
 * 128 x 128 tile of R_g is computed as n_mod residue GEMMs of length
 * d_grp_kdim[g] (multiple of 128, <= 3456) on the tensor cores, CRT-recombined
 * in FP64 from digits merged over consecutive moduli pairs with the HOST
 * constants pair_inv (m_2p^-1 mod m_2p+1) and per-digit f_hi/f_lo/M (see
 * atomx_b200/split_plan.py), scaled and corrected, and written (and
 * mirrored) into the n x n block at d_out + d_grp_out[g], as
 * rkb_table_contract_fp64 does.  The FP64 core correction of a 32 x 64 block
 * is skipped when its bound from d_cbound (relative to 2^(e_a + e_b), which
 * the Schwarz scale of every entry exceeds) is <= corr_floor; pass 0 to
 * always apply it.  Device waits are bounded; *d_status (device
 * int, zero on entry) receives RKB_ETIMEDOUT or RKB_ENONFINITE on failure.
 * ------------------------------------------------------------------------- */
int rkb_split_rows(const double *d_Pv, const double *d_Qv, long orb_ld, const long *d_pairs,
                   const long *d_row_pair, const int *d_row_k, long nrows, const double *d_w,
                   int nv, int ng, const double *d_ktab, const long *d_koff, int bits, int n_mod,
                   const int *moduli, signed char *d_resA, signed char *d_resB, long kpad,
                   long row_base, long nrows_total, double *d_rowscale, double *d_left,
                   double *d_right, double *d_cbound, int cwp, double *d_xwork,
                   const int *d_zcount, void *stream);

/* rkb_split_rows_fused: the rkb_split_rows computation in one kernel that
 * keeps each row in registers (no FP64 workspace), for grids whose body fits:
 * 5 <= ng <= 11, ceil((nv-1)/floor(32/ng)) <= 32 passes, at most max_z <= 64
 * Z columns per multipole (the largest d_zcount).  Residue columns are stored
 * in a fixed permutation shared by every row (the GEMMs are unchanged by it):
 * with cpp = floor(32/ng), body column (m-1)*ng + node of cell m >= 1 is held
 * in pass p = (nv-1-m) / cpp by lane l = ((nv-1-m) % cpp)*ng + node and goes
 * to position 128*(p/4) + 4*l + (p%4); positions of lanes without a cell hold
 * 0; Z column e goes to position rkb_split_fused_body_width(nv, ng) + e.
 * Positions from there + nZ up to kpad are not written (keep them zero).
 * kpad >= body width + max_z.  Scales, core vectors and bounds as in
 * rkb_split_rows. */
int rkb_split_rows_fused(const double *d_Pv, const double *d_Qv, long orb_ld, const long *d_pairs,
                         const long *d_row_pair, const int *d_row_k, long nrows, const double *d_w,
                         int nv, int ng, const double *d_ktab, const long *d_koff, int max_z, int bits,
                         int n_mod, const int *moduli, signed char *d_resA, signed char *d_resB,
                         long kpad, long row_base, long nrows_total, double *d_rowscale,
                         double *d_left, double *d_right, double *d_cbound, int cwp, void *stream);

/* rkb_split_rows_cells: the rkb_split_rows computation with one block per
 * row and one thread per cell (5 <= ng <= 11, nv + max_z <= 256 threads,
 * max_z <= 128), no FP64 workspace; residue columns in natural order
 * ((m-1)*ng + node, then Z), positions from (nv-1)*ng + nZ up to kpad
 * written as zeros.  Besides the packed tables (d_ktab/d_koff) it reads a
 * cell-minor copy of each multipole's factors at d_ktab_t + d_koff_t[k]:
 * u[ng][nv] | C[ng][nv] | L[ng][ng][nv] (L[i][node][cell]).
 * Scales, core vectors and bounds as rkb_split_rows. */
int rkb_split_rows_cells(const double *d_Pv, const double *d_Qv, long orb_ld, const long *d_pairs,
                         const long *d_row_pair, const int *d_row_k, long nrows, const double *d_w,
                         int nv, int ng, const double *d_ktab, const long *d_koff,
                         const double *d_ktab_t, const long *d_koff_t, int max_z, int bits,
                         int n_mod, const int *moduli, signed char *d_resA, signed char *d_resB,
                         long kpad, long row_base, long nrows_total, double *d_rowscale,
                         double *d_left, double *d_right, double *d_cbound, int cwp, void *stream);

/* Host-only planning (no device work): the packed factored Green operator of
 * multipole k on the grid r (nv cells x ng nodes, mo/mi the ng x ng partial
 * matrices of atomx numerics/yk.py:65 yk_partial_matrices) with eigenvalue
 * shift threshold tau, in the layout rkb_split_rows reads (d_ktab):
 * u[N] | Lb[nv][ng][ng] | C[nv][ng] | v0[ng] | G00[ng][ng] | sx | nZ |
 * nZ x (cell, z[ng]), sx = r_b^-(k+1)/2 r_l^-k/2 (r_l the last core node,
 * r_b the first body node).  Writes at most cap doubles to out; returns the count
 * written or a negative rkb_status.  atomx has no counterpart (its Y^k is
 * a scan, numerics/yk.py:88; this factors the same operator). */
long rkb_green_factor(const double *r, int nv, int ng, int k, double tau, const double *mo,
                      const double *mi, double *out, long cap);

/* Host-only planning: the factor tables of every multipole ks[0..nk)
 * (increasing, <= kmax) on one grid, each as rkb_green_factor writes it,
 * computed on up to nthreads host threads.  flat gets the tables end to end
 * in ks order (koff[k] = start, -1 for k <= kmax not in ks; at most flat_cap
 * doubles), nz[i] the Z-column count of ks[i], and flat_t the cell-minor copy
 * the cell row kernel reads (rkb_split_rows_cells d_ktab_t): per multipole
 * u^T[ng][nv] | C^T[ng][nv] | Lb as [ng][ng][nv] at koff_t[k] (2N + nv ng^2
 * doubles each; at most flat_t_cap).  Returns the doubles written to flat
 * or a negative rkb_status.  No atomx counterpart (see rkb_green_factor). */
long rkb_green_tables(const double *r, int nv, int ng, const int *ks, int nk, double tau, const double *mo,
                      const double *mi, int nthreads, int kmax, double *flat, long flat_cap, long *koff,
                      double *flat_t, long flat_t_cap, long *koff_t, long *nz);

/* Host-only planning: the table plan of an orbital set, sized by the caller.
 * n_shells kappa shells (maximal runs of equal kappa in orbital order) start
 * at shell_start[s] with shell_size[s] orbitals; allowed[b][k] (k <= k_max)
 * marks the multipoles the angular rules allow for shell pair b (pairs i <= j
 * in i-major order).  Writes pairs[n_pairs][2] (a <= c by shell-pair block,
 * a-major inside a block), pair_block[n_pairs], and the rows (pair, k)
 * grouped by k in increasing order, each k's pairs ascending: row_pair and
 * row_k[n_rows].  Returns n_rows or a negative rkb_status when the counts
 * disagree.  Follows the pair and row order of atomx_b200.plan, which orders
 * atomx's exchange_k_range selection (atomx angular rules) into tables. */
long rkb_table_plan(const long *shell_start, const long *shell_size, int n_shells, const unsigned char *allowed,
                    int k_max, long n_pairs, long n_rows, long *pairs, long *pair_block, long *row_pair,
                    long *row_k);

/* Residue positions spanned by the body in rkb_split_rows_fused's layout (a
 * multiple of 128), or -1 for an invalid grid.  Host-only, no device work. */
long rkb_split_fused_body_width(int nv, int ng);

int rkb_split_contract(const signed char *d_resA, const signed char *d_resB, long kpad,
                       long nrows_total, int n_mod, const int *moduli, const int *pair_inv,
                       const double *f_hi,
                       const double *f_lo, double M, const double *d_rowscale,
                       const double *d_left, const double *d_right, const double *d_cbound,
                       double corr_floor, int cw, int cwp,
                       const long *d_grp_row0, const long *d_grp_n, const long *d_grp_kdim,
                       const long *d_grp_out, const int *d_tasks, long n_tasks, double *d_out,
                       int *d_status, void *stream);

/* rkb_split_certify: per table g (rows d_grp_row0[g] .. + d_grp_n[g]) the
 * estimate d_est[g] = max_a h_a / sqrt|R_aa| * max_b |[X|Z]_b| / sqrt|R_bb|
 * of the split's Schwarz-relative error from the row records (h = d_rowscale,
 * rows with [X|Z] = 0 skipped, a vanishing or non-finite diagonal gives inf);
 * *d_flagged (device int, cleared by the call) counts the tables with
 * d_est[g] > limit.  Only the row kernels' output is read, so it may run
 * before or after rkb_split_contract.  atomx has no counterpart: it computes
 * every entry in FP64; the split engine recomputes the flagged tables with
 * the FP64 entry points. */
int rkb_split_certify(const long *d_grp_row0, const long *d_grp_n, long n_groups, const double *d_rowscale,
                      const double *d_cbound, double limit, double *d_est, int *d_flagged, void *stream);

/* ---------------------------------------------------------------------------
 * Cell (bank) R^k engine: atomx numerics/bspline/convol.py (the DBSR_HF cell
 * algorithm of the CI, MBPT and Dirac-Fock Fock-matrix paths).
 *
 * A bank of one component pair (left x, right y, orders ks_l, ks_r) holds
 * rkb[i][j][ip][jp] (convol.py:1507 ConvolCache.get_rkb); on the device it is
 * stored as the matrix K[(ip*ns + i)][(jp*ns + j)] = rkb[i][j][ip][jp] at a
 * (row, column) offset of a caller-owned block matrix of leading dimension ld.
 * Moments are (kk, nv) with kk = ks (ks+1)/2 packed upper pairs (i <= j);
 * diagonal cells are (kk_l, kk_r, nv).  Banks built this way equal atomx's
 * bit for bit.
 *
 * rkb_gauss_legendre_01: host only; the n-point Gauss-Legendre rule on [0, 1]
 *   by Newton's iteration on the Legendre recurrence (convol.py:253
 *   _gauss_legendre_01), the sub-quadrature of the diagonal cells.
 * rkb_cell_moments: sum_m grw gr^k B_i B_j per cell, k < 0 meaning
 *   grw / gr^-k (convol.py:58 _compute_moments_sym); bsp is (nv, ng, ks).
 * rkb_cell_diag: the diagonal-cell integrals with an n_sub-point inner rule
 *   (x01, w01 on [0, 1]): same != 0 is _triang_sym (convol.py:136, knots t_l =
 *   t_r), same == 0 is _triang_pqpq (convol.py:388).
 * rkb_cell_assemble: the bank from the left/right rising (r^k) and falling
 *   (r^-(k+1)) moments and the diagonal cells (convol.py:324, :533).
 * rkb_cell_densities: banded pair densities of _density_sym (convol.py:713)
 *   for pairs (d_pairs[2p], d_pairs[2p+1]) of rows of c1, c2 (stored lengths
 *   n1, n2 <= ld; extent ns_d <= ns_k) into out[p*out_ld + col_off + s*ns_k + i].
 * rkb_gemm_nt_fp64: C (+)= A B^T in FP64 on the DMMA pipe (K a multiple of 16,
 *   A and B 16-byte aligned with even leading dimensions): the pair potentials
 *   W = D K^T of batched cell integrals (convol.py:2084) and the table GEMMs
 *   of compute_slater_rk_table (convol.py:1988).
 * rkb_cell_dots: out[e] = L[il[e]] . W[iw[e]] over n columns (one integral
 *   per entry: the trace of _sum_amb_banded, convol.py:1349).
 * rkb_cell_exchange: _convol_case4_t (convol.py:1001) for nbatch densities
 *   (ns x ns each) on the bank blocks at K + kofs[b]; symmetric computes the
 *   lower triangle and mirrors it; accumulate adds into out.
 * rkb_cell_bilinear: _rkb_bilinear (convol.py:1901) on one bank block: T
 *   scratch (ns_out * n_right * ks_r doubles) and M (ns_out x ns_out).
 * rkb_cell_direct_density / rkb_cell_exchange_density: the density sums of
 *   DFSolver._build_hf_matrix_dbsr (methods/dirac_fock.py:1128 with
 *   convol.py:647 / :689) for nbatch coefficient rows (coef + b*coef_stride):
 *   banded (ks x ns rows at out + b*out_ld, source j = target[b] doubled) and
 *   full (ns x ns).
 * rkb_cell_banded_to_full: V[i][i+s] += v[s*ns + i] and its mirror
 *   (convol.py:815 _banded_to_full_add), nbatch (v, V) pairs.
 * rkb_cell_fock_finish: the symmetrisation and norm division closing
 *   _build_hf_matrix_dbsr (dirac_fock.py:1295-1319) on nbatch sets of
 *   (PP, QQ, PQ, QP) blocks; out must not alias h.
 * ------------------------------------------------------------------------- */
void rkb_gauss_legendre_01(int n, double *x, double *w);
int rkb_cell_moments(const double *d_bsp, const double *d_gr, const double *d_grw, int nv, int ng, int ks, int k,
                     double *d_out, void *stream);
int rkb_cell_diag(const double *d_bsp_l, const double *d_bsp_r, const double *d_gr, const double *d_grw,
                  const double *d_t_l, const double *d_t_r, int nv, int ng, int ks_l, int ks_r, int same, int k,
                  const double *d_x01, const double *d_w01, int n_sub, double *d_out, void *stream);
int rkb_cell_assemble(const double *d_rising_l, const double *d_falling_l, const double *d_rising_r,
                      const double *d_falling_r, const double *d_diag, int nv, int ks_l, int ks_r, int ns,
                      double *d_out, long ld, long row_off, long col_off, void *stream);
int rkb_cell_densities(const double *d_c1, const double *d_c2, long ld, const long *d_pairs, long n_pairs, int n1,
                       int n2, int ns_d, int ns_k, int ks, double *d_out, long out_ld, long col_off, void *stream);
int rkb_gemm_nt_fp64(const double *d_A, long lda, const double *d_B, long ldb, double *d_C, long ldc, long M, long N,
                     long K, int accumulate, void *stream);
int rkb_cell_dots(const double *d_L, long l_ld, const double *d_W, long w_ld, long n, const long *d_il,
                  const long *d_iw, long n_ent, double *d_out, void *stream);
int rkb_cell_exchange(const double *d_K, long ld, const long *d_kofs, const double *d_dens, long nbatch, int ns,
                      int ks_l, int ks_r, int symmetric, int accumulate, double *d_out, void *stream);
int rkb_cell_bilinear(const double *d_K, long ld, int ns, const double *d_wa, const double *d_wb, int n_left,
                      int n_right, int ks_l, int ks_r, int ns_out, double *d_T, double *d_M, void *stream);
int rkb_cell_direct_density(const double *d_comp, long ld, int n_orb, const double *d_coef, long coef_stride,
                            const int *d_target, long nbatch, int ns, int ks, double *d_out, long out_ld,
                            void *stream);
int rkb_cell_exchange_density(const double *d_comp_ii, const double *d_comp_jj, long ld, int n_orb,
                              const double *d_coef, long coef_stride, long nbatch, int ns, double *d_out,
                              void *stream);
int rkb_cell_banded_to_full(const double *d_v, int ns, int ks, long nbatch, double *d_V, void *stream);
int rkb_cell_fock_finish(const double *d_h, const double *d_norm, int ns, int skip_pq, long nbatch, double *d_out,
                         void *stream);

/* ---------------------------------------------------------------------------
 * rkb_split_rows_noalloc: no counterpart in the reference (an addition of this
 * library).  The same computation and arguments as rkb_split_rows, without
 * d_xwork: the FP64 row workspace is a fixed device array inside the library,
 * so the call allocates no device memory.  For hosts that cannot allocate on
 * this path (a C or Fortran program with its own device pool that links only
 * this ABI; a process that plans all device memory up front and cannot let
 * cudaMalloc / cudaFree synchronise the device mid-pipeline).
 *
 * Limit: (row_base + nrows) * kpad <= RKB_SPLIT_ROWS_NOALLOC_MAX_DOUBLES
 * (16 MiB of doubles, held on every GPU that loads the library until exit);
 * larger requests return RKB_EINVAL.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current;
 * make it before any stream capture.  The address is kept for the life of the
 * process, so the library must not be used across a cudaDeviceReset of that
 * device.  All calls share the array: calls that overlap on the GPU race, so
 * serialise them.
 * ------------------------------------------------------------------------- */
#define RKB_SPLIT_ROWS_NOALLOC_MAX_DOUBLES (2L * 1024L * 1024L)

int rkb_split_rows_noalloc(const double *d_Pv, const double *d_Qv, long orb_ld, const long *d_pairs,
                           const long *d_row_pair, const int *d_row_k, long nrows, const double *d_w,
                           int nv, int ng, const double *d_ktab, const long *d_koff, int bits, int n_mod,
                           const int *moduli, signed char *d_resA, signed char *d_resB, long kpad,
                           long row_base, long nrows_total, double *d_rowscale, double *d_left,
                           double *d_right, double *d_cbound, int cwp, const int *d_zcount,
                           void *stream);

#ifdef __cplusplus
}
#endif

#endif /* RKB200_H */
