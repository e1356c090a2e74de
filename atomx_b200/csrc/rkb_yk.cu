// Y^k screening functions, orbital values, pair densities, quadrature dots and
// the direct O(N^2) integrator — all FP64 on CUDA cores.
//
// Y^k rule (atomx numerics/yk.py:88-154): with g_j = w_j rho_j on the cell
// Gauss grid,
//     I_out(i in cell m) = A_m + sum_{j in m} g_j r_j^k      mo[i][j]
//     I_in (i in cell m) = B_m + sum_{j in m} g_j r_j^-(k+1) mi[i][j]
//     Y_i = r_i^-(k+1) I_out(i) + r_i^k I_in(i)
// where A_m (B_m) is the sum of g r^k (g r^-(k+1)) over all cells left
// (right) of m.  One warp owns one row: lane l owns cell 32c+l of chunk c,
// forms its cell's terms in registers, and the cell bases come from a
// warp-shuffle scan plus a running carry across chunks.  Within a cell every
// product and sum is evaluated in the reference's order with round-to-nearest
// intrinsics (no FMA contraction), so the only difference from the serial
// reference is the association order of the cross-cell base sums.
#include <cstdarg>
#include <mutex>
#include <map>
#include <utility>
#include <vector>

#include "rkb_common.cuh"

namespace rkb {

// ------------------------------------------------------------------- errors
static thread_local char g_err[512] = "no error";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_status(cudaError_t err, const char *what) {
    set_error("CUDA error in %s: %s (%s)", what, cudaGetErrorName(err), cudaGetErrorString(err));
    return RKB_ECUDA;
}

cudaError_t set_smem_once(const void *func, int bytes) {
    // the attribute only ever grows, so a smaller request never undoes a larger one
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    int &cur = limit[std::make_pair(func, dev)];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

int sm_count() {
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

// ------------------------------------------------------------ Y^k kernels
// Density source for a row: either an explicit row or a pair of orbitals.
// ``row(q)`` resolves a row's source pointers once; ``at(i)`` reads node i.
struct RhoRows {
    const double *rho;
    long ld;
    struct Row {
        const double *__restrict__ rho;
        __device__ __forceinline__ double at(long i) const { return __ldg(rho + i); }
    };
    __device__ __forceinline__ Row row(long q) const { return Row{rho + q * ld}; }
};
struct RhoPairs {
    const double *P, *Q;
    long orb_ld;
    const long *pairs, *row_pair;
    struct Row {
        const double *__restrict__ pa, *__restrict__ pc, *__restrict__ qa, *__restrict__ qc;
        // rho = P_a P_c + Q_a Q_c (atomx slater_yk.py:193), each product rounded
        __device__ __forceinline__ double at(long i) const {
            return __dadd_rn(__dmul_rn(__ldg(pa + i), __ldg(pc + i)), __dmul_rn(__ldg(qa + i), __ldg(qc + i)));
        }
    };
    __device__ __forceinline__ Row row(long q) const {
        const long p = row_pair[q];
        const long a = pairs[2 * p], c = pairs[2 * p + 1];
        return Row{P + a * orb_ld, P + c * orb_ld, Q + a * orb_ld, Q + c * orb_ld};
    }
};

// One warp per row; NG is the compile-time node count (0 = runtime ng <= RKB_MAX_NG).
// `gout` (optional) receives g = w*rho for the row (table engine), and columns
// n..ld-1 of both outputs are zero-filled.
//
// Each pass walks the row in chunks of 32 cells.  The element-wise work of a
// chunk (rho, g, the powers of r, the output Y) runs with consecutive lanes on
// consecutive nodes, so every global load and store is coalesced; the
// per-cell terms meet the cell-owning lane through a per-warp buffer of
// 32 cells x GS doubles (GS = ng | 1: odd stride, no bank conflicts), and the
// cell sums, the warp scan and the partial-matrix sums run as before, lane l
// owning one cell.  I_out waits in the output row between the passes.  Every
// product and sum is the one the cell-per-lane form evaluates, in the same
// order, so the rows are bit-identical to it.
template <int NG, class Src>
__global__ void __launch_bounds__(128) yk_rows_kernel(Src src, const int *__restrict__ row_k, int k_all, long nrows,
                                                      const double *__restrict__ r, const double *__restrict__ w,
                                                      int nv, int ng_rt, const double *__restrict__ mo,
                                                      const double *__restrict__ mi, double *__restrict__ yk,
                                                      long yk_ld, double *__restrict__ gout) {
    constexpr int NGMAX = NG > 0 ? NG : RKB_MAX_NG;
    constexpr int GSMAX = NGMAX | 1;
    const int ng = NG > 0 ? NG : ng_rt;
    const int gs = NG > 0 ? (NG | 1) : (ng_rt | 1);
    extern __shared__ double smem_chunk[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const long n = (long)nv * ng;
    double *cbuf = smem_chunk + (long)wib * (32 * GSMAX);  // [32][gs]: one chunk's per-node terms
    const long q = (long)blockIdx.x * (blockDim.x >> 5) + wib;
    if (q >= nrows) return;
    const int k = row_k ? row_k[q] : k_all;
    const int nchunks = (nv + 31) >> 5;
    const auto sr = src.row(q);  // the row's source pointers, resolved once
    double *yrow = yk + q * yk_ld;
    double *grow_ = gout ? gout + q * yk_ld : nullptr;

    // ---- outward pass: A_m carried left to right; lane l owns cell 32c + l
    double carry = 0.0;
    for (int c = 0; c < nchunks; ++c) {
        const int m0 = c << 5;
        const int ncell = min(32, nv - m0);
        const long e0 = (long)m0 * ng, ne = (long)ncell * ng;
        // element-wise: h = (w rho) r^k, consecutive lanes on consecutive nodes
        for (long t = lane; t < ne; t += 32) {
            const long i = e0 + t;
            const double g = __dmul_rn(__ldg(w + i), sr.at(i));
            if (grow_) grow_[i] = g;
            const int cl = (int)(t / ng), node = (int)(t - (long)cl * ng);
            cbuf[cl * gs + node] = __dmul_rn(g, int_pow(__ldg(r + i), k));
        }
        __syncwarp();
        const int m = m0 + lane;
        const bool live = m < nv;
        double h[NGMAX];
        double cell = 0.0;
        if (live) {
#pragma unroll
            for (int j = 0; j < NGMAX; ++j) {
                if (j < ng) {
                    h[j] = cbuf[lane * gs + j];
                    cell = __dadd_rn(cell, h[j]);
                }
            }
        }
        double incl = warp_inclusive_scan(live ? cell : 0.0, lane);
        double excl = __shfl_up_sync(0xffffffffu, incl, 1);
        double base = lane == 0 ? carry : __dadd_rn(carry, excl);
        carry = __dadd_rn(carry, __shfl_sync(0xffffffffu, incl, 31));
        if (live) {
#pragma unroll
            for (int i = 0; i < NGMAX; ++i) {
                if (i < ng) {
                    double s = base;
#pragma unroll
                    for (int j = 0; j < NGMAX; ++j)
                        if (j < ng) s = __dadd_rn(s, __dmul_rn(h[j], __ldg(&mo[i * ng + j])));
                    cbuf[lane * gs + i] = s;  // own slots only: h is in registers
                }
            }
        }
        __syncwarp();
        // I_out parked in the output row (coalesced); the inward pass reads it
        // back and overwrites it with Y
        for (long t = lane; t < ne; t += 32) {
            const int cl = (int)(t / ng), node = (int)(t - (long)cl * ng);
            yrow[e0 + t] = cbuf[cl * gs + node];
        }
        __syncwarp();  // cbuf is rewritten by the next chunk
    }
    // ---- inward pass: B_m carried right to left; lane l owns cell (end - l)
    carry = 0.0;
    for (int c = 0; c < nchunks; ++c) {
        const int mhi = nv - 1 - (c << 5);             // cell of lane 0
        const int mlo = max(0, mhi - 31);               // lowest cell of the chunk
        const long e0 = (long)mlo * ng, ne = (long)(mhi - mlo + 1) * ng;
        // element-wise: r^-(k+1) (kept in registers for Y) and e = (w rho) r^-(k+1)
        double rin[NGMAX];
#pragma unroll
        for (int u = 0; u < NGMAX; ++u) {
            const long t = lane + 32L * u;
            if (u < ng && t < ne) {
                const long i = e0 + t;
                const double g = __dmul_rn(__ldg(w + i), sr.at(i));
                rin[u] = int_pow(__ldg(r + i), -(k + 1));
                const int cl = (int)(t / ng), node = (int)(t - (long)cl * ng);
                cbuf[cl * gs + node] = __dmul_rn(g, rin[u]);
            }
        }
        __syncwarp();
        const int m = mhi - lane;
        const bool live = m >= 0;
        const int cl_m = m - mlo;  // this lane's cell in the chunk buffer
        double e[NGMAX];
        double cell = 0.0;
        if (live) {
#pragma unroll
            for (int j = 0; j < NGMAX; ++j) {
                if (j < ng) {
                    e[j] = cbuf[cl_m * gs + j];
                    cell = __dadd_rn(cell, e[j]);
                }
            }
        }
        double incl = warp_inclusive_scan(live ? cell : 0.0, lane);
        double excl = __shfl_up_sync(0xffffffffu, incl, 1);
        double base = lane == 0 ? carry : __dadd_rn(carry, excl);
        carry = __dadd_rn(carry, __shfl_sync(0xffffffffu, incl, 31));
        // I_in of this lane's cell back into its buffer slots (each lane reads
        // and writes only its own cell's slots)
        if (live) {
#pragma unroll
            for (int i = 0; i < NGMAX; ++i) {
                if (i < ng) {
                    double s = base;
#pragma unroll
                    for (int j = 0; j < NGMAX; ++j)
                        if (j < ng) s = __dadd_rn(s, __dmul_rn(e[j], __ldg(&mi[i * ng + j])));
                    cbuf[cl_m * gs + i] = s;
                }
            }
        }
        __syncwarp();
        // element-wise: Y = r^-(k+1) I_out + r^k I_in, coalesced
#pragma unroll
        for (int u = 0; u < NGMAX; ++u) {
            const long t = lane + 32L * u;
            if (u < ng && t < ne) {
                const long i = e0 + t;
                const int cl = (int)(t / ng), node = (int)(t - (long)cl * ng);
                yrow[i] = __dadd_rn(__dmul_rn(rin[u], yrow[i]), __dmul_rn(int_pow(__ldg(r + i), k), cbuf[cl * gs + node]));
            }
        }
        __syncwarp();  // cbuf is rewritten by the next chunk
    }
    // zero padding columns
    for (long i = n + lane; i < yk_ld; i += 32) {
        yrow[i] = 0.0;
        if (grow_) grow_[i] = 0.0;
    }
}

template <class Src>
static int launch_yk(Src src, const int *d_row_k, int k_all, long nrows, const double *d_r, const double *d_w, int nv,
                     int ng, const double *d_mo, const double *d_mi, double *d_yk, long yk_ld, double *d_g,
                     cudaStream_t st) {
    const int warps = 4;
    // the kernel's GSMAX: ng | 1 for the compiled node counts below, RKB_MAX_NG | 1 otherwise
    const bool compiled = (ng >= 2 && ng <= 13) || ng == 16 || ng == 17;
    const int gsmax = compiled ? (ng | 1) : (RKB_MAX_NG | 1);
    const size_t smem = (size_t)warps * 32 * gsmax * sizeof(double);  // one chunk buffer per warp, any grid length
    dim3 grid((unsigned)ceil_div(nrows, warps)), block(32 * warps);
#define RKB_YK_CASE(NGV)                                                                                  \
    case NGV: {                                                                                           \
        auto kern = yk_rows_kernel<NGV, Src>;                                                             \
        RKB_CUDA(set_smem(kern, (int)smem));     \
        kern<<<grid, block, smem, st>>>(src, d_row_k, k_all, nrows, d_r, d_w, nv, ng, d_mo, d_mi, d_yk,   \
                                        yk_ld, d_g);                                                      \
        break;                                                                                            \
    }
    switch (ng) {
        RKB_YK_CASE(2) RKB_YK_CASE(3) RKB_YK_CASE(4) RKB_YK_CASE(5) RKB_YK_CASE(6) RKB_YK_CASE(7)
        RKB_YK_CASE(8) RKB_YK_CASE(9) RKB_YK_CASE(10) RKB_YK_CASE(11) RKB_YK_CASE(12) RKB_YK_CASE(13)
        RKB_YK_CASE(16) RKB_YK_CASE(17)
        default: {
            auto kern = yk_rows_kernel<0, Src>;
            RKB_CUDA(set_smem(kern, (int)smem));
            kern<<<grid, block, smem, st>>>(src, d_row_k, k_all, nrows, d_r, d_w, nv, ng, d_mo, d_mi, d_yk, yk_ld,
                                            d_g);
        }
    }
#undef RKB_YK_CASE
    RKB_LAUNCHED("yk_rows_kernel");
    return RKB_OK;
}

static int check_grid(int nv, int ng, long n) {
    RKB_CHECK_ARG(nv >= 1 && ng >= 1 && ng <= RKB_MAX_NG, "need nv >= 1 and 1 <= ng <= %d (got nv=%d ng=%d)",
                  RKB_MAX_NG, nv, ng);
    RKB_CHECK_ARG(n == (long)nv * ng, "n=%ld must equal nv*ng=%ld", n, (long)nv * ng);
    return RKB_OK;
}

// ------------------------------------------------------------ orbital values
__global__ void eval_orbitals_kernel(const double *__restrict__ coeff, long coeff_ld, long n_orb,
                                     const double *__restrict__ bsp, int nv, int ng, int ks, int ns,
                                     double *__restrict__ out, long out_ld) {
    long n = (long)nv * ng;
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * n_orb) return;
    long o = t / n, node = t % n;
    int iv = (int)(node / ng);
    const double *b = bsp + node * ks;
    double s = 0.0;
    for (int j = 0; j < ks; ++j) {
        int gi = iv + j;
        double c = gi < ns ? coeff[o * coeff_ld + gi] : 0.0;
        s = __dadd_rn(s, __dmul_rn(c, b[j]));
    }
    out[o * out_ld + node] = s;
}

__global__ void pair_density_kernel(const double *__restrict__ P, const double *__restrict__ Q, long orb_ld,
                                    const long *__restrict__ pairs, long n_pairs, long n,
                                    double *__restrict__ rho, long rho_ld) {
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * n_pairs) return;
    long p = t / n, i = t % n;
    long a = pairs[2 * p], c = pairs[2 * p + 1];
    rho[p * rho_ld + i] = __dadd_rn(__dmul_rn(P[a * orb_ld + i], P[c * orb_ld + i]),
                                    __dmul_rn(Q[a * orb_ld + i], Q[c * orb_ld + i]));
}

// Row i of a symmetric n x n table, entries j >= i, to the packed upper
// triangle: packed[i*n - i(i-1)/2 + (j - i)].  One block per row.
__global__ void pack_upper_kernel(const double *__restrict__ T, long n, double *__restrict__ packed) {
    const long i = blockIdx.x;
    const double *src = T + i * n;
    double *dst = packed + i * n - (i * (i - 1)) / 2 - i;
    for (long j = i + threadIdx.x; j < n; j += blockDim.x) dst[j] = src[j];
}

// One warp per entry: sum_i (w_i a_i) b_i.
__global__ void weighted_dots_kernel(const double *__restrict__ a, long a_ld, const double *__restrict__ b,
                                     long b_ld, const double *__restrict__ w, long n, const long *__restrict__ ia,
                                     const long *__restrict__ ib, long n_ent, double *__restrict__ out) {
    long e = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (e >= n_ent) return;
    const double *x = a + ia[e] * a_ld, *y = b + ib[e] * b_ld;
    double s = 0.0;
    for (long i = lane; i < n; i += 32) s = __dadd_rn(s, __dmul_rn(__dmul_rn(w[i], x[i]), y[i]));
    s = warp_sum(s);
    if (lane == 0) out[e] = s;
}

// --------------------------------------------------------- direct integrator
// Single block: every thread accumulates a strided share of the disjoint-cell
// double sum and of the coincident-cell triangle rules; one deterministic
// block reduction at the end.
__global__ void __launch_bounds__(1024) slater_direct_kernel(
        const double *__restrict__ f, const double *__restrict__ g, const double *__restrict__ r,
        const double *__restrict__ w, int nv, int ng, int k, int order, double xi0, const double *__restrict__ x,
        const double *__restrict__ wx, const double *__restrict__ outer, const double *__restrict__ inner,
        double *__restrict__ out) {
    __shared__ double red[32];
    const long n = (long)nv * ng;
    double acc = 0.0;
    // disjoint cells: i in cell m, j in any later cell
    for (long i = threadIdx.x; i < n; i += blockDim.x) {
        long j0 = (i / ng + 1) * ng;
        double ri = r[i], wi = w[i], fi = f[i], gi = g[i];
        double part = 0.0;
        for (long j = j0; j < n; ++j) {
            double rj = r[j];
            double ker = int_pow(ri / rj, k) / rj;
            part += w[j] * ker * (fi * g[j] + f[j] * gi);
        }
        acc += wi * part;
    }
    // coincident cells: lower triangle r = a + h x, s = a + h x y
    const long tri = (long)nv * order * order;
    for (long t = threadIdx.x; t < tri; t += blockDim.x) {
        int cidx = (int)(t / (order * order));
        int ix = (int)((t / order) % order), iy = (int)(t % order);
        const double *rc = r + (long)cidx * ng, *wc = w + (long)cidx * ng;
        const double *fc = f + (long)cidx * ng, *gc = g + (long)cidx * ng;
        double h = 0.0;
        for (int m = 0; m < ng; ++m) h += wc[m];
        // cell left edge from its first node: a = r_0 - h (1 + xi_0) / 2
        double aa = rc[0] - h * (1.0 + xi0) / 2.0;
        double xx = x[ix], yy = x[iy];
        double rr = aa + h * xx, ss = aa + h * xx * yy;
        double kj = int_pow(ss / rr, k) / rr * h * h * xx;
        double fo = 0.0, go = 0.0, fi = 0.0, gi = 0.0;
        const double *ov = outer + (long)ix * ng, *iv = inner + ((long)ix * order + iy) * ng;
        for (int m = 0; m < ng; ++m) {
            fo += fc[m] * ov[m];
            go += gc[m] * ov[m];
            fi += fc[m] * iv[m];
            gi += gc[m] * iv[m];
        }
        acc += (fo * gi + go * fi) * kj * wx[ix] * wx[iy];
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) out[0] = v;
    }
}

}  // namespace rkb

using namespace rkb;

extern "C" {

const char *rkb_last_error(void) { return g_err; }

const char *rkb_version(void) { return "rkb200 0.1.0 (sm_100a)"; }

int rkb_device_supported(void) {
    int dev = 0, major = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) return 0;
    return major == 10 ? 1 : 0;
}

// The output rows hold I_out between the kernel's two passes, so they must not
// overlap the density rows the second pass reads again.
static bool overlaps(const double *a, long a_rows, long a_ld, const double *b, long b_rows, long b_ld, long n) {
    const double *a1 = a + (a_rows - 1) * a_ld + n, *b1 = b + (b_rows - 1) * b_ld + n;
    return a < b1 && b < a1;
}

int rkb_yk_flat(const double *d_rho, const double *d_r, const double *d_w, long n, int k, int nv, int ng,
                const double *d_mo, const double *d_mi, double *d_yk, void *stream) {
    int st = check_grid(nv, ng, n);
    if (st) return st;
    RKB_CHECK_ARG(k >= 0 && k <= 64, "multipole rank must be an integer in [0, 64] (got %d)", k);
    RKB_CHECK_ARG(!overlaps(d_rho, 1, n, d_yk, 1, n, n), "d_yk must not overlap d_rho");
    return launch_yk(RhoRows{d_rho, n}, nullptr, k, 1, d_r, d_w, nv, ng, d_mo, d_mi, d_yk, n, nullptr,
                     as_stream(stream));
}

int rkb_yk_rows(const double *d_rho, long rho_ld, const int *d_row_k, long nrows, const double *d_r,
                const double *d_w, int nv, int ng, const double *d_mo, const double *d_mi, double *d_yk,
                long yk_ld, void *stream) {
    long n = (long)nv * ng;
    int st = check_grid(nv, ng, n);
    if (st) return st;
    RKB_CHECK_ARG(nrows >= 0, "nrows must be >= 0");
    RKB_CHECK_ARG(rho_ld >= n && yk_ld >= n, "leading dimensions must be >= nv*ng");
    if (nrows == 0) return RKB_OK;
    RKB_CHECK_ARG(!overlaps(d_rho, nrows, rho_ld, d_yk, nrows, yk_ld, n), "d_yk must not overlap d_rho");
    return launch_yk(RhoRows{d_rho, rho_ld}, d_row_k, 0, nrows, d_r, d_w, nv, ng, d_mo, d_mi, d_yk, yk_ld, nullptr,
                     as_stream(stream));
}

int rkb_table_rows_fp64(const double *d_Pv, const double *d_Qv, long orb_ld, const long *d_pairs,
                        const long *d_row_pair, const int *d_row_k, long nrows, const double *d_r,
                        const double *d_w, int nv, int ng, const double *d_mo, const double *d_mi, double *d_g,
                        double *d_y, long ld, void *stream) {
    long n = (long)nv * ng;
    int st = check_grid(nv, ng, n);
    if (st) return st;
    RKB_CHECK_ARG(ld >= n && orb_ld >= n, "leading dimensions must be >= nv*ng");
    if (nrows == 0) return RKB_OK;
    return launch_yk(RhoPairs{d_Pv, d_Qv, orb_ld, d_pairs, d_row_pair}, d_row_k, 0, nrows, d_r, d_w, nv, ng, d_mo,
                     d_mi, d_y, ld, d_g, as_stream(stream));
}

int rkb_eval_orbitals(const double *d_coeff, long coeff_ld, long n_orb, const double *d_bsp, int nv, int ng,
                      int ks, int ns, double *d_out, long out_ld, void *stream) {
    RKB_CHECK_ARG(nv >= 1 && ng >= 1 && ks >= 1 && ns >= 1, "invalid basis sizes");
    RKB_CHECK_ARG(coeff_ld >= ns && out_ld >= (long)nv * ng, "invalid leading dimensions");
    long total = (long)nv * ng * n_orb;
    if (total == 0) return RKB_OK;
    eval_orbitals_kernel<<<(unsigned)ceil_div(total, 256), 256, 0, as_stream(stream)>>>(
        d_coeff, coeff_ld, n_orb, d_bsp, nv, ng, ks, ns, d_out, out_ld);
    RKB_LAUNCHED("eval_orbitals_kernel");
    return RKB_OK;
}

int rkb_pair_density(const double *d_P, const double *d_Q, long orb_ld, const long *d_pairs, long n_pairs, long n,
                     double *d_rho, long rho_ld, void *stream) {
    RKB_CHECK_ARG(n >= 1 && orb_ld >= n && rho_ld >= n, "invalid sizes");
    long total = n * n_pairs;
    if (total == 0) return RKB_OK;
    pair_density_kernel<<<(unsigned)ceil_div(total, 256), 256, 0, as_stream(stream)>>>(d_P, d_Q, orb_ld, d_pairs,
                                                                                       n_pairs, n, d_rho, rho_ld);
    RKB_LAUNCHED("pair_density_kernel");
    return RKB_OK;
}

int rkb_pack_upper(const double *d_table, long n, double *d_packed, void *stream) {
    RKB_CHECK_ARG(n >= 0 && n <= 0x7fffffffL, "invalid table size %ld", n);
    if (n == 0) return RKB_OK;
    pack_upper_kernel<<<(unsigned)n, 256, 0, as_stream(stream)>>>(d_table, n, d_packed);
    RKB_LAUNCHED("pack_upper_kernel");
    return RKB_OK;
}

int rkb_weighted_dots(const double *d_a, long a_ld, const double *d_b, long b_ld, const double *d_w, long n,
                      const long *d_ia, const long *d_ib, long n_ent, double *d_out, void *stream) {
    RKB_CHECK_ARG(n >= 1 && a_ld >= n && b_ld >= n, "invalid sizes");
    if (n_ent == 0) return RKB_OK;
    weighted_dots_kernel<<<(unsigned)ceil_div(n_ent, 8), 256, 0, as_stream(stream)>>>(d_a, a_ld, d_b, b_ld, d_w, n,
                                                                                     d_ia, d_ib, n_ent, d_out);
    RKB_LAUNCHED("weighted_dots_kernel");
    return RKB_OK;
}

int rkb_slater_direct(const double *d_rho13, const double *d_rho24, const double *d_r, const double *d_w, int nv,
                      int ng, int k, int order, double xi0, const double *d_x, const double *d_wx, const double *d_outer,
                      const double *d_inner, double *d_out, void *stream) {
    RKB_CHECK_ARG(nv >= 1 && ng >= 1 && order >= 1, "invalid sizes");
    RKB_CHECK_ARG(k >= 0 && k <= 64, "multipole rank must be an integer in [0, 64] (got %d)", k);
    slater_direct_kernel<<<1, 1024, 0, as_stream(stream)>>>(d_rho13, d_rho24, d_r, d_w, nv, ng, k, order, xi0, d_x, d_wx,
                                                           d_outer, d_inner, d_out);
    RKB_LAUNCHED("slater_direct_kernel");
    return RKB_OK;
}

}  // extern "C"
