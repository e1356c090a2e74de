// Plain FP64 table contraction: R_g = G_g Y_g^T for every multipole group g,
// where row i of G_g is w*rho of the group's i-th pair and row j of Y_g is
// Y^k of its j-th pair (the slater_rk_poisson sum of atomx
// numerics/bspline/slater.py:130 evaluated for a whole table at once).
//
// The table is symmetric in (ac)<->(bd), so only 128x128 tiles with
// tile_j >= tile_i are computed; off-diagonal tiles are stored twice (as
// computed and transposed).  Arithmetic is FP64 on the FP64 tensor pipe
// (mma.sync m8n8k4 .f64 — sm_100a has no FP64 tcgen05 kind), operands staged
// through shared memory by a 3-deep cp.async ring.  One persistent CTA per SM
// walks a host-built task list (group, tile_i, tile_j).
#include "rkb_common.cuh"
#include "rkb_dmma.cuh"

namespace rkb {
namespace fp64tab {

constexpr int BM = 128, BN = 128, BK = 16, PAD = 4, LDS = BK + PAD, STAGES = 3;
constexpr int THREADS = 256;  // 8 warps as 2 (M) x 4 (N); warp tile 64 x 32
constexpr size_t SMEM = (size_t)STAGES * (BM + BN) * LDS * sizeof(double);


// Stage rows [row0, row0+128) x cols [k0, k0+BK) of a row-major (nrows x ld)
// matrix into smem (128 x LDS); rows past nrows are zero-filled.
__device__ __forceinline__ void load_tile(double *s, const double *__restrict__ g, long ld, long row0, long nrows,
                                          long k0) {
    // 128 rows x 16 doubles = 1024 chunks of 16 B; 4 per thread
#pragma unroll
    for (int it = 0; it < 4; ++it) {
        int c = threadIdx.x + it * THREADS;
        int row = c >> 3, col = (c & 7) * 2;
        long grow = row0 + row;
        bool ok = grow < nrows;
        const double *src = g + (ok ? grow : row0) * ld + k0 + col;
        cp_async16(s + row * LDS + col, src, ok ? 16 : 0);
    }
}

__global__ void __launch_bounds__(THREADS, 1)
contract_kernel(const double *__restrict__ G, const double *__restrict__ Y, long ld, long kdim,
                const long *__restrict__ grp_kdim, const long *__restrict__ grp_row0, const long *__restrict__ grp_n,
                const long *__restrict__ grp_out, const int *__restrict__ tasks, long n_tasks,
                double *__restrict__ out) {
    extern __shared__ double smem[];
    double *As = smem;
    double *Bs = smem + STAGES * BM * LDS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp >> 2, wn = warp & 3;
    const int fr = lane >> 2, fc = lane & 3;
    for (long t = blockIdx.x; t < n_tasks; t += gridDim.x) {
        const int g = tasks[3 * t], ti = tasks[3 * t + 1], tj = tasks[3 * t + 2];
        const int nk = (int)((grp_kdim ? grp_kdim[g] : kdim) / BK);
        const long row0 = grp_row0[g], n = grp_n[g];
        const long i0 = (long)ti * BM, j0 = (long)tj * BN;
        const double *Ag = G + row0 * ld, *Bg = Y + row0 * ld;

        double acc[8][4][2];
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

        __syncthreads();  // previous task's readers are done with the ring
#pragma unroll
        for (int s = 0; s < STAGES - 1; ++s) {
            if (s < nk) {
                load_tile(As + s * BM * LDS, Ag, ld, i0, n, (long)s * BK);
                load_tile(Bs + s * BN * LDS, Bg, ld, j0, n, (long)s * BK);
            }
            cp_async_commit();
        }
        for (int kb = 0; kb < nk; ++kb) {
            cp_async_wait<STAGES - 2>();
            __syncthreads();
            int pf = kb + STAGES - 1;
            if (pf < nk) {
                int s = pf % STAGES;
                load_tile(As + s * BM * LDS, Ag, ld, i0, n, (long)pf * BK);
                load_tile(Bs + s * BN * LDS, Bg, ld, j0, n, (long)pf * BK);
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

        double *R = out + grp_out[g];
        const bool mirror = tj != ti;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            long i = i0 + wm * 64 + a * 8 + fr;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                long j = j0 + wn * 32 + b * 8 + fc * 2;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    if (i < n && j + e < n) {
                        R[i * n + j + e] = acc[a][b][e];
                        if (mirror) R[(j + e) * n + i] = acc[a][b][e];
                    }
                }
            }
        }
    }
}

}  // namespace fp64tab
}  // namespace rkb

using namespace rkb;

static int launch_contract(const double *d_g, const double *d_y, long ld, long kdim, const long *d_grp_kdim,
                           const long *d_grp_row0, const long *d_grp_n, const long *d_grp_out, const int *d_tasks,
                           long n_tasks, double *d_out, void *stream) {
    if (n_tasks == 0) return RKB_OK;
    auto kern = fp64tab::contract_kernel;
    RKB_CUDA(set_smem(kern, (int)fp64tab::SMEM));
    long grid = n_tasks < sm_count() ? n_tasks : sm_count();
    kern<<<(unsigned)grid, fp64tab::THREADS, fp64tab::SMEM, as_stream(stream)>>>(
        d_g, d_y, ld, kdim, d_grp_kdim, d_grp_row0, d_grp_n, d_grp_out, d_tasks, n_tasks, d_out);
    RKB_LAUNCHED("fp64tab::contract_kernel");
    return RKB_OK;
}

extern "C" int rkb_table_contract_fp64(const double *d_g, const double *d_y, long ld, long kdim,
                                       const long *d_grp_row0, const long *d_grp_n, const long *d_grp_out,
                                       const int *d_tasks, long n_tasks, double *d_out, void *stream) {
    RKB_CHECK_ARG(kdim >= 0 && kdim % fp64tab::BK == 0 && ld >= kdim && ld % 2 == 0,
                  "contraction length %ld must be a multiple of %d and <= ld (%ld, even)", kdim, fp64tab::BK, ld);
    return launch_contract(d_g, d_y, ld, kdim, nullptr, d_grp_row0, d_grp_n, d_grp_out, d_tasks, n_tasks, d_out,
                           stream);
}

extern "C" int rkb_table_contract_fp64_groups(const double *d_g, const double *d_y, long ld, long max_kdim,
                                              const long *d_grp_kdim, const long *d_grp_row0, const long *d_grp_n,
                                              const long *d_grp_out, const int *d_tasks, long n_tasks,
                                              double *d_out, void *stream) {
    RKB_CHECK_ARG(d_grp_kdim != nullptr, "per-group contraction lengths are required");
    RKB_CHECK_ARG(max_kdim >= 0 && ld >= max_kdim && ld % 2 == 0, "contraction lengths must be <= ld (%ld, even)",
                  ld);
    return launch_contract(d_g, d_y, ld, max_kdim, d_grp_kdim, d_grp_row0, d_grp_n, d_grp_out, d_tasks, n_tasks,
                           d_out, stream);
}
