// Arbitrary-grid trapezoid Y^k on the device (atomx numerics/quadrature.py).
//
// atomx's yk_on_grid / yk_pair_dot_batch_on_grid (quadrature.py:234-372) act
// with the Coulomb Green kernel r_<^k / r_>^(k+1) on a density sampled on an
// arbitrary increasing grid, by two cumulative trapezoid scans in
// block-scaled frames: within frame b the tables hold rk_i = (r_i/a_b)^k and
// inverse_i = (r_i/a_b)^-(k+1) / a_b, and a carried moment changes frame by
// the factor transfer[b] = (a_b / a_(b+1))^k <= 1 (quadrature.py:190-231).
//
//   inward:  acc_i = sum over intervals j >= i of 0.5 (b_j + b_(j+1)) dr_j,
//            b_j = rho_j inverse_j, rescaled by transfer at each frame
//            change; y_i = acc_i (y_(n-1) = 0)
//   outward: inner_i = sum over intervals j <= i of 0.5 (a_(j-1) + a_j) dr,
//            a_j = rho_j rk_j, likewise rescaled;
//            y_i = inner_i inverse_i + rk_i y_i,  y_0 = y_0 rk_0
//
// The reference runs both scans serially per row.  Here one CTA owns a row:
// each frame is scanned in tiles of TILE points with a block-wide exclusive
// prefix (outward) or suffix (inward) sum, formed without subtractions (a
// difference of partial sums would cancel on grids whose terms grow along
// the row), and the carry between tiles and frames is kept in shared memory
// and rescaled exactly where the reference rescales it.  Rows are independent (persistent CTAs walk the row list).  The
// summation order inside a frame differs from the serial one, so results
// agree with the reference to rounding, not bit for bit.
#include "rkb_common.cuh"

namespace rkb {
namespace grid {

constexpr int THREADS = 256;
constexpr int ITEMS = 4;
constexpr int TILE = THREADS * ITEMS;

struct Tables {
    const double *r, *rk, *inverse;  // rk / inverse: the row's multipole, n values
    const long *cuts;                // frame starts, ncuts values (cuts[ncuts-1] = n)
    long ncuts;
    const double *transfer;          // the row's multipole, ncuts-2 values
    long n, i_cut;
};

// Density of a row: either a sampled rho, or P_a P_b + Q_a Q_b formed on the
// fly (quadrature.py:313-352 forms it in the same way).
struct Dens {
    const double *rho, *Pa, *Qa, *Pb, *Qb;
    __device__ __forceinline__ double operator()(long i) const {
        return rho ? rho[i] : __dadd_rn(__dmul_rn(Pa[i], Pb[i]), __dmul_rn(Qa[i], Qb[i]));
    }
};

// Block-wide exclusive scan of one double per thread (sum over lower
// threadIdx), formed without subtracting: the lane below's inclusive value
// plus the totals of the lower warps.  *total receives the block's sum.
__device__ __forceinline__ double block_scan_excl(double v, double *sh, double *total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double incl = warp_inclusive_scan(v, lane);
    const double below = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 31) sh[wid] = incl;
    __syncthreads();
    double before = 0.0, all = 0.0;
    for (int w = 0; w < nw; ++w) {
        if (w < wid) before += sh[w];
        all += sh[w];
    }
    __syncthreads();
    *total = all;
    return lane == 0 ? before : before + below;
}

__device__ __forceinline__ double block_total(double v, double *sh) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    __syncthreads();
    return t;
}

// Both scans of one row; y (i_cut + 1 values) receives the result.
__device__ void row_scan(const Tables &T, const Dens &rho, double *y, double *sh) {
    const long n = T.n, ic = T.i_cut;
    const int t = threadIdx.x;
    double *carry = sh + 32;
    // ---- inward, frames from the top; intervals j in [cuts[b], min(cuts[b+1]-1, n-2)]
    if (t == 0) *carry = 0.0;
    if (ic == n - 1 && t == 0) y[n - 1] = 0.0;
    __syncthreads();
    for (long b = T.ncuts - 2; b >= 0; --b) {
        const long lo = T.cuts[b];
        const long hi = T.cuts[b + 1] - 1 < n - 2 ? T.cuts[b + 1] - 1 : n - 2;  // top interval of the frame
        if (b < T.ncuts - 2) {
            if (t == 0) *carry *= T.transfer[b];
            __syncthreads();
        }
        for (long top = hi; top >= lo; top -= TILE) {
            // thread t handles intervals top - ITEMS*t - s, s = 0..ITEMS-1 (descending)
            double term[ITEMS];
            double local = 0.0;
#pragma unroll
            for (int s = 0; s < ITEMS; ++s) {
                const long j = top - (long)ITEMS * t - s;
                term[s] = 0.0;
                if (j >= lo) {
                    const double bj = rho(j) * T.inverse[j];
                    double bn = rho(j + 1) * T.inverse[j + 1];
                    if (j + 1 == T.cuts[b + 1] && b < T.ncuts - 2) bn *= T.transfer[b];
                    term[s] = .5 * (bj + bn) * (T.r[j + 1] - T.r[j]);
                }
                local += term[s];
            }
            double tile;
            const double above = block_scan_excl(local, sh, &tile);  // intervals above this thread's
            const double c0 = *carry;
            double run = c0 + above;
#pragma unroll
            for (int s = 0; s < ITEMS; ++s) {
                const long j = top - (long)ITEMS * t - s;
                run += term[s];
                if (j >= lo && j <= ic) y[j] = run;
            }
            __syncthreads();
            if (t == 0) *carry = c0 + tile;
            __syncthreads();
        }
    }
    __syncthreads();
    // ---- outward, frames from the bottom; points i in [max(1, cuts[b]), min(cuts[b+1], ic+1))
    if (t == 0) {
        *carry = 0.0;
        y[0] *= T.rk[0];
    }
    __syncthreads();
    for (long b = 0; b < T.ncuts - 1; ++b) {
        if (T.cuts[b] > ic) break;
        if (b) {
            if (t == 0) *carry *= T.transfer[b - 1];
            __syncthreads();
        }
        const long lo = T.cuts[b] > 1 ? T.cuts[b] : 1;
        const long hi = T.cuts[b + 1] < ic + 1 ? T.cuts[b + 1] : ic + 1;
        for (long base = lo; base < hi; base += TILE) {
            double term[ITEMS];
            double local = 0.0;
#pragma unroll
            for (int s = 0; s < ITEMS; ++s) {
                const long i = base + (long)ITEMS * t + s;
                term[s] = 0.0;
                if (i < hi) {
                    const double ai = rho(i) * T.rk[i];
                    double ap = rho(i - 1) * T.rk[i - 1];
                    if (i == T.cuts[b] && b > 0) ap *= T.transfer[b - 1];
                    term[s] = .5 * (ai + ap) * (T.r[i] - T.r[i - 1]);
                }
                local += term[s];
            }
            double tile;
            const double below = block_scan_excl(local, sh, &tile);  // points below this thread's
            const double c0 = *carry;
            double run = c0 + below;
#pragma unroll
            for (int s = 0; s < ITEMS; ++s) {
                const long i = base + (long)ITEMS * t + s;
                run += term[s];
                if (i < hi) y[i] = run * T.inverse[i] + T.rk[i] * y[i];
            }
            __syncthreads();
            if (t == 0) *carry = c0 + tile;
            __syncthreads();
        }
    }
    __syncthreads();
}

struct BatchArgs {
    const double *PA, *QA, *PB, *QB, *rho;
    long ld, rho_ld;
    const long *rows_a, *rows_b, *rows_k;
    const unsigned char *rows_ok;
    long nrows;
    const double *W;  // consumer weight rows (ld w_ld), or null: write y instead
    long w_ld;
    const long *cons_ptr, *cons_rho;
    const double *r, *RK, *inverse, *transfers;
    const long *cuts;
    long n, ncuts, ntr, i_cut;
    double *val;        // consumer dots
    double *y, *work;   // y rows (ld y_ld) when W is null, else work rows (one per CTA)
    long y_ld;
};

__global__ void __launch_bounds__(THREADS) grid_rows_kernel(BatchArgs a) {
    __shared__ double sh[40];
    for (long m = blockIdx.x; m < a.nrows; m += gridDim.x) {
        if (a.rows_ok && !a.rows_ok[m]) continue;
        const bool dots = a.W != nullptr;
        if (dots && a.cons_ptr[m] == a.cons_ptr[m + 1]) continue;
        const long k = a.rows_k[m];
        Tables T{a.r, a.RK + k * a.n, a.inverse + k * a.n, a.cuts, a.ncuts, a.transfers + k * a.ntr, a.n, a.i_cut};
        Dens d{nullptr, nullptr, nullptr, nullptr, nullptr};
        if (a.rho) {
            d.rho = a.rho + m * a.rho_ld;
        } else {
            d.Pa = a.PA + a.rows_a[m] * a.ld;
            d.Qa = a.QA + a.rows_a[m] * a.ld;
            d.Pb = a.PB + a.rows_b[m] * a.ld;
            d.Qb = a.QB + a.rows_b[m] * a.ld;
        }
        double *y = dots ? a.work + (long)blockIdx.x * a.n : a.y + m * a.y_ld;
        row_scan(T, d, y, sh);
        if (!dots) continue;
        for (long s = a.cons_ptr[m]; s < a.cons_ptr[m + 1]; ++s) {
            const double *w = a.W + a.cons_rho[s] * a.w_ld;
            double part = 0.0;
            for (long i = threadIdx.x; i <= a.i_cut; i += blockDim.x) part = fma(w[i], y[i], part);
            const double tot = block_total(part, sh);
            if (threadIdx.x == 0) a.val[s] = tot;
        }
        __syncthreads();
    }
}

}  // namespace grid
}  // namespace rkb

using namespace rkb;

static int grid_common_checks(long n, long ncuts, long ntr, long i_cut) {
    RKB_CHECK_ARG(n >= 1, "empty grid");
    RKB_CHECK_ARG(ncuts >= 2 && ntr >= ncuts - 2, "invalid frame tables (ncuts=%ld, transfers=%ld)", ncuts, ntr);
    RKB_CHECK_ARG(i_cut >= 0 && i_cut <= n - 1, "i_cut %ld outside [0, %ld]", i_cut, n - 1);
    return RKB_OK;
}

extern "C" int rkb_grid_yk_rows(const double *d_rho, long rho_ld, const long *d_rows_k, long nrows,
                                const double *d_r, long n, const double *d_RK, const double *d_inverse,
                                const long *d_cuts, long ncuts, const double *d_transfers, long ntr, long i_cut,
                                double *d_y, long y_ld, void *stream) {
    int st = grid_common_checks(n, ncuts, ntr, i_cut);
    if (st != RKB_OK) return st;
    RKB_CHECK_ARG(y_ld >= n && rho_ld >= n, "row strides must be >= n");
    if (nrows == 0) return RKB_OK;
    grid::BatchArgs a = {};
    a.rho = d_rho; a.rho_ld = rho_ld; a.rows_k = d_rows_k; a.nrows = nrows;
    a.r = d_r; a.RK = d_RK; a.inverse = d_inverse; a.transfers = d_transfers; a.cuts = d_cuts;
    a.n = n; a.ncuts = ncuts; a.ntr = ntr; a.i_cut = i_cut; a.y = d_y; a.y_ld = y_ld;
    const long grid_n = nrows < 8L * sm_count() ? nrows : 8L * sm_count();
    grid::grid_rows_kernel<<<(unsigned)grid_n, grid::THREADS, 0, as_stream(stream)>>>(a);
    RKB_LAUNCHED("grid_rows_kernel");
    return RKB_OK;
}

extern "C" int rkb_grid_pair_dot_batch(const double *d_PA, const double *d_QA, const double *d_PB,
                                       const double *d_QB, long ld, const long *d_rows_a, const long *d_rows_b,
                                       const long *d_rows_k, const unsigned char *d_rows_ok, long nrows,
                                       const double *d_W, long w_ld, const long *d_cons_ptr,
                                       const long *d_cons_rho, const double *d_r, long n, const double *d_RK,
                                       const double *d_inverse, const long *d_cuts, long ncuts,
                                       const double *d_transfers, long ntr, long i_cut, double *d_val,
                                       double *d_work, long work_rows, void *stream) {
    int st = grid_common_checks(n, ncuts, ntr, i_cut);
    if (st != RKB_OK) return st;
    RKB_CHECK_ARG(ld >= n && w_ld >= i_cut + 1, "row strides too small (ld=%ld, w_ld=%ld)", ld, w_ld);
    RKB_CHECK_ARG(d_work != nullptr && work_rows >= 1, "a work area of at least one row is required");
    if (nrows == 0) return RKB_OK;
    grid::BatchArgs a = {};
    a.PA = d_PA; a.QA = d_QA; a.PB = d_PB; a.QB = d_QB; a.ld = ld; a.rows_a = d_rows_a; a.rows_b = d_rows_b;
    a.rows_k = d_rows_k; a.rows_ok = d_rows_ok; a.nrows = nrows; a.W = d_W; a.w_ld = w_ld;
    a.cons_ptr = d_cons_ptr; a.cons_rho = d_cons_rho; a.r = d_r; a.RK = d_RK; a.inverse = d_inverse;
    a.transfers = d_transfers; a.cuts = d_cuts; a.n = n; a.ncuts = ncuts; a.ntr = ntr; a.i_cut = i_cut;
    a.val = d_val; a.work = d_work;
    const long grid_n = nrows < work_rows ? nrows : work_rows;
    grid::grid_rows_kernel<<<(unsigned)grid_n, grid::THREADS, 0, as_stream(stream)>>>(a);
    RKB_LAUNCHED("grid_rows_kernel");
    return RKB_OK;
}
