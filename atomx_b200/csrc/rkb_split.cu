// Split-precision R^k engine: factored Green operator + Ozaki-II (CRT) INT8
// residue GEMMs on the 5th-generation tensor cores, recombined in FP64.
//
//   R(ac;bd) = X_ac . X_bd - Z_ac . Z_bd + left_ac . right_bd
//
// K2x  split_rows_kernel  (one warp per (pair, k) row, FP64 on CUDA cores)
//      g = w (P_a P_c + Q_a Q_c);  per body cell m >= 1:  d_m = u_m . g_m and
//      the exclusive suffix sums T_m = sum_{m'>m} d_m' (warp-shuffle scans);
//      X_m = L_mm^T g_m + c_m T_m;  Z_e = z_e . g_{cell(e)};
//      FP64 core terms left = [g_0, alpha sx, q/sx], right = [G_00 g_0, q/sx,
//      alpha sx] with alpha = v_0.g_0 and q = T_0 (the core-body coupling).
//      The FP64 row [X | Z] goes to a scratch buffer with its power-of-two
//      scale (|x| < 2^bits); split_residues_kernel then rounds it to integers
//      x~ and writes int8 residues x~ mod m_i (and the B copy with Z negated)
//      in a [modulus][row][kpad] layout, one 16-byte store per modulus.
//      Per row the kernels also record (cbound, CB_STRIDE doubles): the
//      screen bounds |g_0|, |G_00 g_0|, |alpha sx|, |q/sx| relative to the row
//      scale, and for the certificate |[X | Z]| and the FP64 diagonal
//      R_aa = |X|^2 - |Z|^2 + left.right.
//
// K3s  crt_syrk_kernel  (persistent, one CTA per SM, 18 warps)
//      warp 0: TMA producer — 128x128-byte boxes (SWIZZLE_128B) of the A and B
//              residue matrices into a STAGES-deep ring;
//      warp 1: TMEM owner + MMA issuer — tcgen05.mma.kind::i8, M=N=128, K=32,
//              int32 accumulators in a double-buffered TMEM tile;
//      warps 2-17: epilogue (4 TMEM lane quarters x 4 column groups; four
//              warps per SM sub-partition hide the TMEM and ALU latency) — per
//              modulus: TMEM -> registers, reduce to [0, m) with integer
//              operations, merge each even/odd pair of moduli into a 16-bit
//              digit mod m_e m_o (two digits per 32-bit word; words of four
//              moduli parked in TMEM columns 256..511, the last word kept in
//              registers); per tile: CRT over the digits in FP64 (exact split
//              constants), scale, add the core correction when it is not
//              screened out, store the tile and its transpose.
//      Every mbarrier wait is bounded; on timeout the kernel records
//      RKB_ETIMEDOUT in *status and every role drains and returns.
#include <cuda.h>

#include <cfloat>

#include <mutex>

#include "rkb_common.cuh"

namespace rkb {
namespace split {

constexpr int MAXMOD = 12;
// Doubles per row of the cbound array: [0] |g_0|, [1] |G_00 g_0|, [2] |alpha sx|,
// [3] |q/sx| (each times 2^-e of the row scale), [4] |[X | Z]|, [5] R_aa, [6..7] 0.
constexpr int CB_STRIDE = 8;

// The per-row record: screen bounds relative to 2^-e (infinite for a zero
// row, which is never screened), the row norm and the FP64 diagonal.
__device__ __forceinline__ void write_row_record(double *cb, double amax, int ex, double n_g0, double n_gg,
                                                 double a_sx, double q_sx, double xsq, double zsq, double g0gg) {
    const double rel = amax > 0.0 ? ldexp(1.0, -ex) : INFINITY;
    cb[0] = sqrt(n_g0) * rel;
    cb[1] = sqrt(n_gg) * rel;
    cb[2] = fabs(a_sx) * rel;
    cb[3] = fabs(q_sx) * rel;
    cb[4] = sqrt(xsq + zsq);
    cb[5] = xsq - zsq + g0gg + 2.0 * a_sx * q_sx;
    cb[6] = 0.0;
    cb[7] = 0.0;
}

// =========================================================================
// K2x — transform, quantise, residues
// =========================================================================
struct RowsArgs {
    const double *P, *Q;
    long orb_ld;
    const long *pairs, *row_pair;
    const int *row_k;
    long nrows;
    const double *w;
    int nv, ng;
    const double *ktab;
    const long *koff;  // by k
    int bits, n_mod;
    int mod[MAXMOD];
    uint32_t magic[MAXMOD], c20[MAXMOD], bias[MAXMOD];  // 2^32/m + 1, 2^20 mod m, m * 2^20
    double inv_mod[MAXMOD];    // RN(1/m)
    signed char *resA, *resB;  // [n_mod][nrows_total][kpad]; resB may be null
    long kpad, row_base, nrows_total;
    double *rowscale, *left, *right, *cbound;
    double *xwork;  // scratch rows [X | Z | 0] (row stride kpad)
    int cwp;
};

__device__ __forceinline__ double rho_at(const RowsArgs &a, long q, long i) {
    long p = a.row_pair[q];
    long x = a.pairs[2 * p], c = a.pairs[2 * p + 1];
    return __dadd_rn(__dmul_rn(a.P[x * a.orb_ld + i], a.P[c * a.orb_ld + i]),
                     __dmul_rn(a.Q[x * a.orb_ld + i], a.Q[c * a.orb_ld + i]));
}

// x mod m in [0, m) for 0 <= x < 2^32 with integer operations only:
// q = hi32(x * (floor(2^32/m) + 1)) exceeds x/m by less than x/2^32 < 1, so it
// is floor(x/m) or one more, and one conditional add repairs the remainder.
__device__ __forceinline__ uint32_t umod_small(uint32_t x, uint32_t m, uint32_t magic) {
    const uint32_t q = __umulhi(x, magic);
    int r = (int)(x - q * m);
    return (uint32_t)(r + (r < 0 ? (int)m : 0));
}

// Centred int8 residue (as a byte) of an integer x = hi * 2^20 + lo, |hi| <= 2^20, 0 <= lo < 2^20.
__device__ __forceinline__ uint32_t residue_i8(int hi, uint32_t lo, uint32_t m, uint32_t magic, uint32_t c20,
                                               uint32_t bias) {
    // (hi mod m) * (2^20 mod m) + (lo mod m): every operand nonnegative and < 2^29
    const uint32_t h = umod_small((uint32_t)(hi + (int)bias), m, magic);
    const uint32_t l = umod_small(lo, m, magic);
    const uint32_t r = umod_small(h * c20 + l, m, magic);
    const int rc = (int)r - (r > 127u ? (int)m : 0);
    return (uint32_t)rc & 0xffu;
}

// One warp per row.  Shared memory per warp: g (n doubles) and the per-cell
// suffix sums (nv doubles).  Cells are processed by lane groups of ng lanes
// (lane = node of a cell), so shared and global accesses are consecutive
// across lanes.  The FP64 row [X | Z | 0...] goes to the caller's scratch
// buffer; split_residues_kernel turns it into int8 residues.
template <int NG>
__global__ void __launch_bounds__(128) split_rows_kernel(RowsArgs a) {
    const int ng = NG > 0 ? NG : a.ng;
    const int nv = a.nv;
    const long n = (long)nv * ng;
    extern __shared__ double sm[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    // segment lengths rounded to even counts of doubles keep every segment 16-byte aligned
    const long np = (n + 1) & ~1L, nvp = (nv + 1) & ~1L;
    const long per_warp = np + nvp;
    double *g = sm + (long)wib * per_warp;
    double *tsuf = g + np;
    const long q = (long)blockIdx.x * (blockDim.x >> 5) + wib;
    if (q >= a.nrows) return;
    const int k = a.row_k[q];
    const double *tab = a.ktab + a.koff[k];
    const double *u = tab;
    const double *Lb = u + n;
    const double *C = Lb + (long)nv * ng * ng;
    const double *v0 = C + (long)nv * ng;
    const double *G00 = v0 + ng;
    const double sx = G00[ng * ng];
    const int nz = (int)G00[ng * ng + 1];
    const double *zt = G00 + ng * ng + 2;
    const long kbody = (long)(nv - 1) * ng;
    // lane groups: cpp cells per pass, lane -> (cell offset, node)
    const int cpp = 32 / ng;
    const int sub = lane / ng, node = lane - sub * ng;
    const bool glane = sub < cpp;

    for (long i = lane; i < n; i += 32) g[i] = __dmul_rn(a.w[i], rho_at(a, q, i));
    __syncwarp();
    // alpha = v_0 . g_0: the core multipole moment of the core-body coupling
    double alpha = 0.0;
    for (int j = lane; j < ng; j += 32) alpha = fma(v0[j], g[j], alpha);
    alpha = warp_sum(alpha);

    // cell dots d_m = u_m . g_m (m >= 1) by lane groups, segmented shuffle sums
    for (int m0 = 0; m0 < nv; m0 += cpp) {
        const int m = m0 + sub;
        double p = 0.0;
        if (glane && m >= 1 && m < nv) p = u[(long)m * ng + node] * g[(long)m * ng + node];
        // sum over the ng lanes of the group (groups never straddle: lanes >= cpp*ng idle)
        double tot = 0.0;
        for (int t = 0; t < ng; ++t) tot += __shfl_sync(0xffffffffu, p, sub * ng + t < 32 ? sub * ng + t : lane);
        if (glane && node == 0 && m < nv) tsuf[m] = (m >= 1) ? tot : 0.0;
    }
    __syncwarp();
    // exclusive suffix sums over cells: lane l owns cell (end - l) of each chunk
    const int nch = (nv + 31) >> 5;
    double carry = 0.0;
    for (int c = 0; c < nch; ++c) {
        const int m = nv - 1 - ((c << 5) + lane);
        const double d = m >= 0 ? tsuf[m] : 0.0;
        const double incl = warp_inclusive_scan(d, lane);
        const double excl = __shfl_up_sync(0xffffffffu, incl, 1);
        __syncwarp();
        if (m >= 0) tsuf[m] = lane == 0 ? carry : carry + excl;
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    __syncwarp();

    // the row [X | Z | 0...] into the scratch row, with its maximum and sums of squares
    const long grow = a.row_base + q;  // row index in the residue matrices
    double *xs = a.xwork + grow * a.kpad;
    double amax = 0.0, xsq = 0.0, zsq = 0.0;
    bool bad = false;  // fmax drops NaNs, so non-finite values are tracked apart
    for (int m0 = 1; m0 < nv; m0 += cpp) {
        const int m = m0 + sub;
        if (glane && m < nv) {
            const double *L = Lb + (long)m * ng * ng;
            const double *gm = g + (long)m * ng;
            double x = C[(long)m * ng + node] * tsuf[m];
            for (int i = node; i < ng; ++i) x = fma(L[i * ng + node], gm[i], x);
            xs[(long)(m - 1) * ng + node] = x;
            amax = fmax(amax, fabs(x));
            xsq = fma(x, x, xsq);
            bad |= !isfinite(x);
        }
    }
    for (int e = lane; e < nz; e += 32) {
        const double *ze = zt + (long)e * (ng + 1);
        const double *gm = g + (long)ze[0] * ng;
        double x = 0.0;
        for (int i = 0; i < ng; ++i) x = fma(ze[1 + i], gm[i], x);
        xs[kbody + e] = x;
        amax = fmax(amax, fabs(x));
        zsq = fma(x, x, zsq);
        bad |= !isfinite(x);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    xsq = warp_sum(xsq);
    zsq = warp_sum(zsq);

    for (long c = kbody + nz + lane; c < a.kpad; c += 32) xs[c] = 0.0;
    int ex = 0;
    double inv_scale = 0.0;
    if (amax > 0.0 && isfinite(amax)) {
        frexp(amax, &ex);  // amax < 2^ex
        inv_scale = ldexp(1.0, ex - a.bits);
    }

    // FP64 core terms: left = [g_0, alpha sx, q/sx], right = [G_00 g_0, q/sx, alpha sx]
    const double a_sx = alpha * sx, q_sx = tsuf[0] / sx;  // T_0 = u_b . g_b
    bad |= !isfinite(a_sx) || !isfinite(q_sx);
    double *lf = a.left + grow * a.cwp, *rt = a.right + grow * a.cwp;
    double n1 = 0.0, n2 = 0.0, gg = 0.0;
    for (int i = lane; i < a.cwp; i += 32) {
        double gi = 0.0, sacc = 0.0;
        if (i < ng) {
            gi = g[i];
            for (int j = 0; j < ng; ++j) sacc = fma(G00[i * ng + j], g[j], sacc);
            n1 = fma(gi, gi, n1);
            n2 = fma(sacc, sacc, n2);
            gg = fma(gi, sacc, gg);
        } else if (i == ng) {
            gi = a_sx;
            sacc = q_sx;
        } else if (i == ng + 1) {
            gi = q_sx;
            sacc = a_sx;
        }
        lf[i] = gi;
        rt[i] = sacc;
    }
    n1 = warp_sum(n1);
    n2 = warp_sum(n2);
    gg = warp_sum(gg);
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
        // a non-finite row gets a NaN scale: its residues are zero and every
        // entry it reaches is NaN, which the contraction reports
        a.rowscale[grow] = bad ? __longlong_as_double(0x7ff8000000000000LL) : inv_scale;
        write_row_record(a.cbound + grow * CB_STRIDE, amax, ex, n1, n2, a_sx, q_sx, xsq, zsq, gg);
    }
}


// Residues of the scaled rows: one thread per (row, 16 columns).  x = rint(X *
// 2^(bits - e_row)) is an exact integer with |x| <= 2^bits; each modulus gets
// one 16-byte store (and the B copy negates the row's Z columns).
__global__ void __launch_bounds__(256) split_residues_kernel(RowsArgs a, const int *__restrict__ z_count) {
    const long per_row = a.kpad / 16;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.nrows * per_row) return;
    const long q = t / per_row, c0 = (t - q * per_row) * 16;
    const long grow = a.row_base + q;
    const double rs = a.rowscale[grow];
    const double scale = rs > 0.0 ? 1.0 / rs : 0.0;  // an exact power of two
    const double *xs = a.xwork + grow * a.kpad + c0;
    int hi[16];
    uint32_t lo[16];
#pragma unroll
    for (int j = 0; j < 16; j += 2) {
        const double2 v = *reinterpret_cast<const double2 *>(xs + j);
        double y0 = v.x * scale, y1 = v.y * scale;
        y0 = fabs(y0) <= 0x1p40 ? y0 : 0.0;  // NaN rows (and a zero scale) give zeros
        y1 = fabs(y1) <= 0x1p40 ? y1 : 0.0;
        const long long x0 = (long long)rint(y0), x1 = (long long)rint(y1);
        hi[j] = (int)(x0 >> 20);
        lo[j] = (uint32_t)(x0 & 0xfffffLL);
        hi[j + 1] = (int)(x1 >> 20);
        lo[j + 1] = (uint32_t)(x1 & 0xfffffLL);
    }
    const long kbody = (long)(a.nv - 1) * a.ng;
    const long zhi = kbody + z_count[a.row_k[q]];
    const bool anyz = a.resB != nullptr && c0 + 16 > kbody && c0 < zhi;
    for (int md = 0; md < a.n_mod; ++md) {
        const uint32_t m = (uint32_t)a.mod[md], magic = a.magic[md], c20 = a.c20[md], bias = a.bias[md];
        uint32_t w[4], wb[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            uint32_t va = 0u, vb = 0u;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const int j = 4 * i + s;
                const uint32_t r = residue_i8(hi[j], lo[j], m, magic, c20, bias);
                va |= r << (8 * s);
                uint32_t rb = r;
                if (anyz && c0 + j >= kbody && c0 + j < zhi) {
                    int nr = -(int)(int8_t)(uint8_t)r;  // residue of -x, centred again
                    nr -= nr > 127 ? (int)m : 0;
                    rb = (uint32_t)nr & 0xffu;
                }
                vb |= rb << (8 * s);
            }
            w[i] = va;
            wb[i] = vb;
        }
        const long o = ((long)md * a.nrows_total + grow) * a.kpad + c0;
        *reinterpret_cast<uint4 *>(a.resA + o) = make_uint4(w[0], w[1], w[2], w[3]);
        if (a.resB) *reinterpret_cast<uint4 *>(a.resB + o) = make_uint4(wb[0], wb[1], wb[2], wb[3]);
    }
}


// ---------------------------------------------------------------------------
// Fused row kernel (rows whose body fits in registers): one warp per row, no
// shared memory and no FP64 workspace.  Cells are taken from the last to the
// first in passes of CPP = 32/NG cells (lane = (cell offset, node)), so the
// suffix sums t_m = sum_{m'>m} u_m'.g_m' are a running carry; each lane keeps
// its X value of every pass in registers until the row maximum is known, then
// writes int8 residues directly.
//
// Residue layout (any column order shared by every row of a GEMM leaves the
// products unchanged): the value of pass p held by lane l goes to position
// 128*(p/4) + 4*l + (p%4), so four passes form one 32-bit word per lane and a
// warp stores 128 contiguous bytes per modulus.  Lanes without a cell (l >=
// CPP*NG, or cell 0 / below in the last pass) hold zeros.  The body therefore
// spans fused_body_width() positions; Z column e sits at body_width + e.
__host__ __device__ constexpr int fused_cpp(int ng) { return 32 / ng; }
__host__ __device__ inline long fused_passes(int nv, int ng) { return (nv - 1 + fused_cpp(ng) - 1) / fused_cpp(ng); }
__host__ __device__ inline long fused_body_width(int nv, int ng) { return 128 * ((fused_passes(nv, ng) + 3) / 4); }
constexpr int FUSED_PMAX = 32;  // passes kept in registers (body width <= 1024)
constexpr int FUSED_ZMAX = 64;  // Z columns per row (two per lane)

// Centred residue of an integer-valued double |x| <= 2^40 modulo m <= 256:
// q = round(x/m) with the 1.5*2^52 rounding constant (x*inv_m is within
// 2^-13 of x/m, and x/m is never that close to a half-integer except exactly
// at one, where either rounding is fine), r = x - q*m exactly by one fma,
// |r| <= m/2, then moved into [-128, 127].
__device__ __forceinline__ uint32_t residue_f64(double x, double m, double inv_m) {
    const double rc = 6755399441055744.0;  // 1.5 * 2^52
    const double q = __dadd_rn(__fma_rn(x, inv_m, rc), -rc);
    const double r = __fma_rn(-q, m, x);
    int ri = __double2loint(__dadd_rn(r, rc));
    ri -= ri > 127 ? (int)m : 0;
    return (uint32_t)ri & 0xffu;
}

template <int NG>
__global__ void __launch_bounds__(128) split_rows_fused_kernel(RowsArgs a) {
    constexpr int CPP = 32 / NG;
    constexpr unsigned FULL = 0xffffffffu;
    const int nv = a.nv;
    const int lane = threadIdx.x & 31;
    const long q = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (q >= a.nrows) return;
    const int k = a.row_k[q];
    const long pr = a.row_pair[q];
    const double *Pa = a.P + a.pairs[2 * pr] * a.orb_ld, *Pc = a.P + a.pairs[2 * pr + 1] * a.orb_ld;
    const double *Qa = a.Q + a.pairs[2 * pr] * a.orb_ld, *Qc = a.Q + a.pairs[2 * pr + 1] * a.orb_ld;
    const long n = (long)nv * NG;
    const double *tab = a.ktab + a.koff[k];
    const double *u = tab;
    const double *Lb = u + n;
    const double *C = Lb + (long)nv * NG * NG;
    const double *v0 = C + (long)nv * NG;
    const double *G00 = v0 + NG;
    const double sx = G00[NG * NG];
    const int nz = (int)G00[NG * NG + 1];
    const double *zt = G00 + NG * NG + 2;
    const int sub = lane / NG, node = lane - sub * NG;
    const bool glane = sub < CPP;
    const long grow = a.row_base + q;
    auto gval = [&](long i) {
        return __dmul_rn(a.w[i], __dadd_rn(__dmul_rn(Pa[i], Pc[i]), __dmul_rn(Qa[i], Qc[i])));
    };

    // cell 0: g_0 (lanes < NG), alpha = v_0 . g_0, G_00 g_0 and their norms
    const double g0 = lane < NG ? gval(lane) : 0.0;
    const double alpha = warp_sum(lane < NG ? v0[lane] * g0 : 0.0);
    double sg = 0.0;
#pragma unroll
    for (int j = 0; j < NG; ++j) {
        const double gj = __shfl_sync(FULL, g0, j);
        if (lane < NG) sg = fma(G00[lane * NG + j], gj, sg);
    }
    const double n1 = warp_sum(g0 * g0), n2 = warp_sum(sg * sg), gg = warp_sum(g0 * sg);

    // body passes, last cell first
    const int P = (int)fused_passes(nv, NG);
    double xs[FUSED_PMAX];
    double carry = 0.0, amax = 0.0, xsq = 0.0, zsq = 0.0;
    bool bad = false;
#pragma unroll
    for (int p = 0; p < FUSED_PMAX; ++p) {
        xs[p] = 0.0;
        if (p < P) {
            const int m = nv - 1 - p * CPP - sub;
            const bool ok = glane && m >= 1;
            const long i = (long)m * NG + node;
            const double g = ok ? gval(i) : 0.0;
            double dm = ok ? u[i] * g : 0.0;
            // sum over the NG lanes of the group (every lane of the group gets it)
            {
                double tot = 0.0;
#pragma unroll
                for (int t = 0; t < NG; ++t) tot += __shfl_sync(FULL, dm, (sub * NG + t) & 31);
                dm = tot;
            }
            // carry of the cells already passed plus the higher cells of this pass
            double before = 0.0, all = 0.0;
#pragma unroll
            for (int s = 0; s < CPP; ++s) {
                const double ds = __shfl_sync(FULL, dm, s * NG);
                all += ds;
                before += s < sub ? ds : 0.0;
            }
            const double t = carry + before;
            carry += all;
            const double *L = Lb + (long)m * NG * NG;
            double x = ok ? C[i] * t : 0.0;
#pragma unroll
            for (int ii = 0; ii < NG; ++ii) {
                const double gi = __shfl_sync(FULL, g, (sub * NG + ii) & 31);
                if (ok && ii >= node) x = fma(L[ii * NG + node], gi, x);
            }
            xs[p] = x;
            amax = fmax(amax, fabs(x));
            xsq = fma(x, x, xsq);
            bad |= !isfinite(x);
        }
    }
    // core terms: left = [g_0, alpha sx, q/sx], right = [G_00 g_0, q/sx, alpha sx]
    // (the carry now holds q = u_b . g_b on every lane)
    const double a_sx = alpha * sx, q_sx = carry / sx;
    bad |= !isfinite(a_sx) || !isfinite(q_sx);
    if (lane < a.cwp) {
        a.left[grow * a.cwp + lane] = lane < NG ? g0 : (lane == NG ? a_sx : (lane == NG + 1 ? q_sx : 0.0));
        a.right[grow * a.cwp + lane] = lane < NG ? sg : (lane == NG ? q_sx : (lane == NG + 1 ? a_sx : 0.0));
    }
    // Z columns: lane e and e + 32
    double zx[2] = {0.0, 0.0};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int e = lane + 32 * h;
        if (e < nz) {
            const double *ze = zt + (long)e * (NG + 1);
            const long base = (long)ze[0] * NG;
            double x = 0.0;
            for (int ii = 0; ii < NG; ++ii) x = fma(ze[1 + ii], gval(base + ii), x);
            zx[h] = x;
            amax = fmax(amax, fabs(x));
            zsq = fma(x, x, zsq);
            bad |= !isfinite(x);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(FULL, amax, o));
    xsq = warp_sum(xsq);
    zsq = warp_sum(zsq);
    bad = __any_sync(FULL, bad);
    int ex = 0;
    double scale = 0.0, inv_scale = 0.0;
    if (!bad && amax > 0.0) {
        frexp(amax, &ex);  // amax < 2^ex
        scale = ldexp(1.0, a.bits - ex);
        inv_scale = ldexp(1.0, ex - a.bits);
    }
    if (lane == 0) {
        a.rowscale[grow] = bad ? __longlong_as_double(0x7ff8000000000000LL) : inv_scale;
        write_row_record(a.cbound + grow * CB_STRIDE, amax, ex, n1, n2, a_sx, q_sx, xsq, zsq, gg);
    }

    // quantise in place (exact integers, |x| <= 2^bits) and write residues
    const double rc = 6755399441055744.0;
#pragma unroll
    for (int p = 0; p < FUSED_PMAX; ++p) xs[p] = __dadd_rn(__fma_rn(xs[p], scale, rc), -rc);
    zx[0] = __dadd_rn(__fma_rn(zx[0], scale, rc), -rc);
    zx[1] = __dadd_rn(__fma_rn(zx[1], scale, rc), -rc);
    const long bw = fused_body_width(nv, NG);
    for (int md = 0; md < a.n_mod; ++md) {
        const double m = (double)a.mod[md], inv_m = a.inv_mod[md];
        signed char *rowA = a.resA + ((long)md * a.nrows_total + grow) * a.kpad;
        signed char *rowB = a.resB ? a.resB + ((long)md * a.nrows_total + grow) * a.kpad : nullptr;
#pragma unroll
        for (int j = 0; j < FUSED_PMAX / 4; ++j) {
            if (4 * j < P) {
                uint32_t word = 0u;
#pragma unroll
                for (int s = 0; s < 4; ++s) word |= residue_f64(xs[4 * j + s], m, inv_m) << (8 * s);
                reinterpret_cast<uint32_t *>(rowA + 128 * j)[lane] = word;
                if (rowB) reinterpret_cast<uint32_t *>(rowB + 128 * j)[lane] = word;
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int e = lane + 32 * h;
            if (e < nz) {
                const uint32_t r = residue_f64(zx[h], m, inv_m);
                rowA[bw + e] = (signed char)r;
                if (rowB) {
                    int nr = -(int)(int8_t)(uint8_t)r;  // residue of -x, centred again
                    nr -= nr > 127 ? (int)m : 0;
                    rowB[bw + e] = (signed char)nr;
                }
            }
        }
    }
}


// ---------------------------------------------------------------------------
// Cell-parallel row kernel: one block per row, one thread per cell.  Thread t
// owns cell m = nv-1-t (cells last to first), so a forward exclusive block
// scan of the cell dots u_m.g_m gives each cell its suffix sum t_m directly.
// The block first forms g = w*rho for the whole row with coalesced loads
// (consecutive threads, consecutive nodes) into a padded shared-memory image;
// each thread then reads its cell's g and the cell-minor factor copy
// (entry i of every cell contiguous, so a warp's reads are consecutive) and
// forms X = L_m^T g_m + C_m t_m in registers, without shuffles.
// Threads past the cells compute the Z columns.  After a block maximum fixes
// the row's power-of-two scale, every thread writes its int8 residues into
// per-modulus row images in shared memory, and the block copies them out with
// 16-byte stores.  Columns are in natural order: (m-1)*ng + node, then Z.
//
// Cell-minor factor table of one multipole (doubles), nv cells:
//   u[NG][nv] | C[NG][nv] | L[NG][NG][nv] (L[i][node][m])
constexpr int CELL_ZMAX = 128;  // Z columns per row of the cell kernel (one thread each, nv + Z <= 256)

template <int NG>
__global__ void __launch_bounds__(256) split_rows_cell_kernel(RowsArgs a, const double *__restrict__ ktab_t,
                                                              const long *__restrict__ koff_t) {
    constexpr int GS = NG | 1;  // padded cell stride of the g image (odd: 2-way bank conflicts at most)
    extern __shared__ __align__(16) unsigned char smc[];
    const int nv = a.nv;
    const long q = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarp = blockDim.x >> 5;
    const long kpad = a.kpad;
    const size_t ndbl = ((size_t)nv * GS + 64 + 1) & ~(size_t)1;     // doubles before the images (even: 16-B aligned)
    double *gimg = reinterpret_cast<double *>(smc);                  // [nv][GS]
    double *red = gimg + (size_t)nv * GS;                              // [64] block scratch
    unsigned char *lines = smc + ndbl * sizeof(double);               // [n_mod][kpad]
    unsigned char *zneg = lines + (size_t)a.n_mod * kpad;             // [n_mod][CELL_ZMAX]: B's Z bytes
    const int k = a.row_k[q];
    const long pr = a.row_pair[q];
    const double *Pa = a.P + a.pairs[2 * pr] * a.orb_ld, *Pc = a.P + a.pairs[2 * pr + 1] * a.orb_ld;
    const double *Qa = a.Q + a.pairs[2 * pr] * a.orb_ld, *Qc = a.Q + a.pairs[2 * pr + 1] * a.orb_ld;
    const long n = (long)nv * NG;
    const double *tab = a.ktab + a.koff[k];
    const double *v0 = tab + n + (long)nv * NG * NG + (long)nv * NG;
    const double *G00 = v0 + NG;
    const double sx = G00[NG * NG];
    const int nz = (int)G00[NG * NG + 1];
    const double *zt = G00 + NG * NG + 2;
    const double *tt = ktab_t + koff_t[k];
    const double *ut = tt, *Ct = tt + n, *Lt = tt + 2 * n;
    const long kbody = (long)(nv - 1) * NG;
    const long grow = a.row_base + q;
    // g = w * (P_a P_c + Q_a Q_c) for the whole row, coalesced
    for (long j = tid; j < n; j += blockDim.x) {
        const long cell = j / NG, node = j - cell * NG;
        gimg[cell * GS + node] =
            __dmul_rn(a.w[j], __dadd_rn(__dmul_rn(Pa[j], Pc[j]), __dmul_rn(Qa[j], Qc[j])));
    }
    __syncthreads();
    const int m = nv - 1 - tid;  // this thread's cell (m < 0: a Z column or idle)
    double g[NG], x[NG];
    double d = 0.0;
    if (m >= 0) {
#pragma unroll
        for (int i = 0; i < NG; ++i) g[i] = gimg[(long)m * GS + i];
        if (m >= 1) {
#pragma unroll
            for (int i = 0; i < NG; ++i) d = fma(ut[(long)i * nv + m], g[i], d);
        }
    }
    // cell 0: alpha = v_0 . g_0, G_00 g_0 and their norms (one thread)
    double n1 = 0.0, n2 = 0.0, gg = 0.0, alpha = 0.0;
    if (m == 0) {
#pragma unroll
        for (int i = 0; i < NG; ++i) alpha = fma(v0[i], g[i], alpha);
#pragma unroll
        for (int i = 0; i < NG; ++i) {
            double sacc = 0.0;
#pragma unroll
            for (int j = 0; j < NG; ++j) sacc = fma(G00[i * NG + j], g[j], sacc);
            a.left[grow * a.cwp + i] = g[i];
            a.right[grow * a.cwp + i] = sacc;
            n1 = fma(g[i], g[i], n1);
            n2 = fma(sacc, sacc, n2);
            gg = fma(g[i], sacc, gg);
        }
        for (int i = NG + 2; i < a.cwp; ++i) a.left[grow * a.cwp + i] = a.right[grow * a.cwp + i] = 0.0;
    }
    // exclusive scan of d over threads (= suffix sums over cells)
    const double incl = warp_inclusive_scan(d, lane);
    if (lane == 31) red[wid] = incl;
    __syncthreads();
    double before = 0.0;
    for (int w = 0; w < wid; ++w) before += red[w];
    const double up = __shfl_up_sync(0xffffffffu, incl, 1);
    const double t_m = lane == 0 ? before : before + up;
    double amax = 0.0, xsq = 0.0, zsq = 0.0;
    bool bad = false;
    if (m >= 1) {
#pragma unroll
        for (int node = 0; node < NG; ++node) {
            double xv = Ct[(long)node * nv + m] * t_m;
#pragma unroll
            for (int i = node; i < NG; ++i) xv = fma(Lt[((long)i * NG + node) * nv + m], g[i], xv);
            x[node] = xv;
            amax = fmax(amax, fabs(xv));
            xsq = fma(xv, xv, xsq);
            bad |= !isfinite(xv);
        }
    }
    // cell 0: the core-body coupling columns (t_0 = q = u_b . g_b)
    double a_sx = 0.0, q_sx = 0.0;
    if (m == 0) {
        a_sx = alpha * sx;
        q_sx = t_m / sx;
        bad |= !isfinite(a_sx) || !isfinite(q_sx);
        a.left[grow * a.cwp + NG] = a_sx;
        a.left[grow * a.cwp + NG + 1] = q_sx;
        a.right[grow * a.cwp + NG] = q_sx;
        a.right[grow * a.cwp + NG + 1] = a_sx;
    }
    // Z columns: thread nv + e
    const int e = tid - nv;
    double zx = 0.0;
    if (e >= 0 && e < nz) {
        const double *ze = zt + (long)e * (NG + 1);
        const long cz = (long)ze[0];
#pragma unroll
        for (int i = 0; i < NG; ++i) zx = fma(ze[1 + i], gimg[cz * GS + i], zx);
        amax = fmax(amax, fabs(zx));
        zsq = zx * zx;
        bad |= !isfinite(zx);
    }
    // block maximum, sums of squares and non-finite flag (red[]: 8 warps at most)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    xsq = warp_sum(xsq);
    zsq = warp_sum(zsq);
    const int badw = __any_sync(0xffffffffu, bad);
    __syncthreads();  // red[] reused
    if (lane == 0) {
        red[wid] = amax;
        red[8 + wid] = xsq;
        red[16 + wid] = zsq;
        red[32 + wid] = badw ? 1.0 : 0.0;
    }
    __syncthreads();
    amax = 0.0;
    xsq = 0.0;
    zsq = 0.0;
    bool anybad = false;
    for (int w = 0; w < nwarp; ++w) {
        amax = fmax(amax, red[w]);
        xsq += red[8 + w];
        zsq += red[16 + w];
        anybad |= red[32 + w] != 0.0;
    }
    int ex = 0;
    double scale = 0.0, inv_scale = 0.0;
    if (!anybad && amax > 0.0) {
        frexp(amax, &ex);  // amax < 2^ex
        scale = ldexp(1.0, a.bits - ex);
        inv_scale = ldexp(1.0, ex - a.bits);
    }
    if (m == 0) {
        a.rowscale[grow] = anybad ? __longlong_as_double(0x7ff8000000000000LL) : inv_scale;
        write_row_record(a.cbound + grow * CB_STRIDE, amax, ex, n1, n2, a_sx, q_sx, xsq, zsq, gg);
    }
    // residues into the row images (natural column order), zero tails
    const double rc = 6755399441055744.0;  // 1.5 * 2^52
    const long zend = kbody + nz;
    for (long c = zend + tid; c < kpad; c += blockDim.x)
        for (int md = 0; md < a.n_mod; ++md) lines[(size_t)md * kpad + c] = 0;
    if (m >= 1) {
#pragma unroll
        for (int node = 0; node < NG; ++node) x[node] = __dadd_rn(__fma_rn(x[node], scale, rc), -rc);
        for (int md = 0; md < a.n_mod; ++md) {
            const double mm = (double)a.mod[md], im = a.inv_mod[md];
            unsigned char *ln = lines + (size_t)md * kpad + (long)(m - 1) * NG;
#pragma unroll
            for (int node = 0; node < NG; ++node) ln[node] = (unsigned char)residue_f64(x[node], mm, im);
        }
    }
    if (e >= 0 && e < nz) {
        zx = __dadd_rn(__fma_rn(zx, scale, rc), -rc);
        for (int md = 0; md < a.n_mod; ++md) {
            const uint32_t r = residue_f64(zx, (double)a.mod[md], a.inv_mod[md]);
            lines[(size_t)md * kpad + kbody + e] = (unsigned char)r;
            int nr = -(int)(int8_t)(uint8_t)r;  // residue of -x, centred again
            nr -= nr > 127 ? a.mod[md] : 0;
            zneg[md * CELL_ZMAX + e] = (unsigned char)nr;
        }
    }
    __syncthreads();
    // copy the row images out: 16-byte chunks; B's chunks that hold Z columns
    // take their bytes from the negated copy
    const long chunks = kpad / 16;
    const long zc0 = kbody / 16, zc1 = (zend + 15) / 16;
    for (long it = tid; it < (long)a.n_mod * chunks; it += blockDim.x) {
        const int md = (int)(it / chunks);
        const long ch = it - (long)md * chunks;
        const uint4 v = *reinterpret_cast<const uint4 *>(lines + (size_t)md * kpad + ch * 16);
        const long o = ((long)md * a.nrows_total + grow) * kpad + ch * 16;
        *reinterpret_cast<uint4 *>(a.resA + o) = v;
        if (a.resB) {
            if (nz > 0 && ch >= zc0 && ch < zc1) {
                unsigned char tmp[16];
                *reinterpret_cast<uint4 *>(tmp) = v;
                for (int b = 0; b < 16; ++b) {
                    const long c = ch * 16 + b;
                    if (c >= kbody && c < zend) tmp[b] = zneg[md * CELL_ZMAX + (c - kbody)];
                }
                *reinterpret_cast<uint4 *>(a.resB + o) = *reinterpret_cast<const uint4 *>(tmp);
            } else {
                *reinterpret_cast<uint4 *>(a.resB + o) = v;
            }
        }
    }
}

// =========================================================================
// K3s — tcgen05 INT8 residue SYRK with CRT epilogue
// =========================================================================
constexpr int BM = 128, BN = 128, BKB = 128;  // tile rows, tile cols, K bytes per stage
constexpr int STAGES = 5;
constexpr int STAGE_BYTES = (BM + BN) * BKB;  // 32 KB
constexpr int EPI_WARPS = 16;                 // 4 TMEM lane quarters x 4 column groups
constexpr int EPI_COLS = BN / (EPI_WARPS / 4);  // columns per epilogue thread
constexpr int THREADS = 32 * (2 + EPI_WARPS);
constexpr int STG_LD = 9;   // doubles per staged row (8 + pad)
constexpr size_t SMEM_BYTES = 1024 /*align slack*/ + (size_t)STAGES * STAGE_BYTES +
                              (size_t)EPI_WARPS * 32 * STG_LD * sizeof(double) + 256 /*barriers*/;
constexpr long long WAIT_LIMIT = 4000000000LL;  // clock64 ticks (~2 s)
constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

struct CrtArgs {
    const double *rowscale, *left, *right, *cbound;
    double corr_floor;  // skip the FP64 core correction of a warp block when its bound is below this
    int cwp, cw;
    const long *grp_row0, *grp_n, *grp_kdim, *grp_out;
    const int *tasks;
    long n_tasks, nrows_total;
    double *out;
    int *status;
    int n_mod;
    int mod[MAXMOD];
    uint32_t magic[MAXMOD];   // floor(2^32 / m) + 1
    uint32_t bias[MAXMOD];    // m * 2^18: makes every accumulator nonnegative
    uint32_t pinv[MAXMOD / 2];  // m_2p^-1 mod m_2p+1
    double f_hi[MAXMOD], f_lo[MAXMOD];  // per merged digit
    double M;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false (and status = ETIMEDOUT) after WAIT_LIMIT clock ticks,
// or as soon as another role has recorded a failure.
__device__ __forceinline__ bool mbar_wait_slow(uint64_t *bar, uint32_t parity, int *status) {
    long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (*(volatile int *)status != 0) return false;
        if (clock64() - t0 > WAIT_LIMIT) {
            atomicExch(status, (int)RKB_ETIMEDOUT);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *status) {
    if (mbar_try(bar, parity)) return true;
    return mbar_wait_slow(bar, parity, status);
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tma_load(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);   // start address (16-byte units)
    d |= (uint64_t)1u << 16;                   // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32;         // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1u << 46;                   // descriptor version for sm_100
    d |= (uint64_t)2u << 61;                   // SWIZZLE_128B
    return d;
}
__device__ __forceinline__ void mma_i8(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(dtmem),
        "l"(ad), "l"(bd), "r"(IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t *v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::
            "r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
        "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

template <int NMOD>
__global__ void __launch_bounds__(THREADS, 1)
    crt_syrk_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                    const __grid_constant__ CrtArgs p) {
    constexpr int PARKED = (NMOD - 1) >> 2;  // groups of four moduli parked in TMEM (0..2)
    constexpr int LASTG = PARKED;            // group kept in registers
    constexpr int NDIG = (NMOD + 1) / 2;     // merged CRT digits
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *ring = base;
    double *stage_out = (double *)(ring + (size_t)STAGES * STAGE_BYTES);
    uint64_t *bars = (uint64_t *)(stage_out + EPI_WARPS * 32 * STG_LD);
    uint64_t *full = bars, *empty = bars + STAGES, *accf = bars + 2 * STAGES, *acce = accf + 2;
    uint32_t *tmem_slot = (uint32_t *)(acce + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf[b], 1);
            mbar_init(&acce[b], EPI_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    int *status = p.status;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (long t = blockIdx.x; t < p.n_tasks && ok; t += gridDim.x) {
                const int g = p.tasks[3 * t], ti = p.tasks[3 * t + 1], tj = p.tasks[3 * t + 2];
                const long row0 = p.grp_row0[g];
                const int nk = (int)(p.grp_kdim[g] / BKB);
                for (int md = 0; md < NMOD && ok; ++md) {
                    const int ya = (int)(md * p.nrows_total + row0 + (long)ti * BM);
                    const int yb = (int)(md * p.nrows_total + row0 + (long)tj * BN);
                    for (int kc = 0; kc < nk; ++kc, ++it) {
                        const int s = it % STAGES;
                        const uint32_t ph = (it / STAGES) & 1u;
                        if (!mbar_wait(&empty[s], ph ^ 1u, status)) { ok = false; break; }
                        unsigned char *sa = ring + (size_t)s * STAGE_BYTES;
                        mbar_expect_tx(&full[s], STAGE_BYTES);
                        tma_load(sa, &mapA, kc * BKB, ya, &full[s]);
                        tma_load(sa + BM * BKB, &mapB, kc * BKB, yb, &full[s]);
                    }
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            uint32_t it = 0, acc_it = 0;
            bool ok = true;
            for (long t = blockIdx.x; t < p.n_tasks && ok; t += gridDim.x) {
                const int g = p.tasks[3 * t];
                const int nk = (int)(p.grp_kdim[g] / BKB);
                for (int md = 0; md < NMOD && ok; ++md, ++acc_it) {
                    const int buf = acc_it & 1;
                    const uint32_t aph = (acc_it >> 1) & 1u;
                    if (!mbar_wait(&acce[buf], aph ^ 1u, status)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t dt = tmem + (uint32_t)(buf * BN);
                    for (int kc = 0; kc < nk; ++kc, ++it) {
                        const int s = it % STAGES;
                        const uint32_t ph = (it / STAGES) & 1u;
                        if (!mbar_wait(&full[s], ph, status)) { ok = false; break; }
                        tc_fence_after();
                        const uint32_t sa = smem_u32(ring + (size_t)s * STAGE_BYTES);
                        const uint64_t ad = sw128_desc(sa), bd = sw128_desc(sa + BM * BKB);
#pragma unroll
                        for (int kk = 0; kk < BKB / 32; ++kk)
                            mma_i8(dt, ad + (uint64_t)(2 * kk), bd + (uint64_t)(2 * kk), (kc | kk) != 0 ? 1u : 0u);
                        mma_commit(&empty[s]);
                    }
                    if (ok) mma_commit(&accf[buf]);
                }
            }
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const int ew = warp - 2;
        const int quarter = warp & 3;       // TMEM lane quarter this warp may access
        const int cgrp = ew >> 2;           // column group of the tile
        const int rloc = quarter * 32 + lane;
        const uint32_t lane_off = (uint32_t)(quarter * 32) << 16;
        const uint32_t col0 = (uint32_t)(cgrp * EPI_COLS);
        double *stg = stage_out + (size_t)ew * 32 * STG_LD;
        uint32_t acc_it = 0;
        bool ok = true;
        for (long t = blockIdx.x; t < p.n_tasks && ok; t += gridDim.x) {
            const int g = p.tasks[3 * t], ti = p.tasks[3 * t + 1], tj = p.tasks[3 * t + 2];
            const long row0 = p.grp_row0[g], n = p.grp_n[g];
            const long a = (long)ti * BM + rloc;  // table row of this thread
            const long b0 = (long)tj * BN + col0;
            uint32_t pk[EPI_COLS];
#pragma unroll
            for (int c = 0; c < EPI_COLS; ++c) pk[c] = 0u;
#pragma unroll 1
            for (int md = 0; md < NMOD; ++md, ++acc_it) {
                const int buf = acc_it & 1;
                const uint32_t aph = (acc_it >> 1) & 1u;
                if (!mbar_wait(&accf[buf], aph, status)) { ok = false; break; }
                tc_fence_after();
                const uint32_t m = (uint32_t)p.mod[md], magic = p.magic[md], bias = p.bias[md];
                const int fsh = 16 * ((md >> 1) & 1);  // 16-bit field of this pair in the word
                if ((md & 1) == 0) {
                    // even modulus: park r_e in its pair field
#pragma unroll
                    for (int c = 0; c < EPI_COLS / 16; ++c) {
                        uint32_t v[16];
                        tmem_ld16(tmem + lane_off + (uint32_t)(buf * BN) + col0 + (uint32_t)(c * 16), v);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 16; ++j) pk[c * 16 + j] |= umod_small(v[j] + bias, m, magic) << fsh;
                    }
                } else {
                    // odd modulus: merge with the parked r_e into a digit mod m_e m_o
                    const uint32_t me = (uint32_t)p.mod[md - 1], inv = p.pinv[md >> 1];
#pragma unroll
                    for (int c = 0; c < EPI_COLS / 16; ++c) {
                        uint32_t v[16];
                        tmem_ld16(tmem + lane_off + (uint32_t)(buf * BN) + col0 + (uint32_t)(c * 16), v);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            const uint32_t ro = umod_small(v[j] + bias, m, magic);
                            const uint32_t word = pk[c * 16 + j];
                            const uint32_t re = (word >> fsh) & 0xffffu;
                            const uint32_t t = umod_small((ro + 2u * m - re) * inv, m, magic);
                            pk[c * 16 + j] = (word & ~(0xffffu << fsh)) | ((re + me * t) << fsh);
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&acce[buf]);
                if ((md & 3) == 3 && (md >> 2) < PARKED) {
                    // park a completed group of four moduli in TMEM columns 256 + 128*group
                    const uint32_t col = 256u + 128u * (uint32_t)(md >> 2) + col0;
#pragma unroll
                    for (int c = 0; c < EPI_COLS / 16; ++c) tmem_st16(tmem + lane_off + col + (uint32_t)(c * 16), &pk[c * 16]);
                    tmem_wait_st();
#pragma unroll
                    for (int c = 0; c < EPI_COLS; ++c) pk[c] = 0u;
                }
            }
            if (!ok) break;
            // ---- CRT, scaling, correction and stores
            const bool arow = a < n;
            const double rs_a = arow ? __ldg(p.rowscale + row0 + a) : 0.0;
            const double *la = p.left + (row0 + (arow ? a : 0)) * p.cwp;
            const bool mirror = ti != tj;
            double *R = p.out + p.grp_out[g];
            // Correction screen for this warp's 32 x EPI_COLS block: with per-row bounds
            // relative to each row's scale, |left_a . right_b| <= 2^(e_a+e_b) *
            // (|g0_a| |G00 g0_b| + |alpha_a sx| |q_b/sx| + |q_a/sx| |alpha_b sx|).
            // Below corr_floor the term is far under the split's own error and is skipped.
            double ra0 = 0.0, ra2 = 0.0, ra3 = 0.0, cb1 = 0.0, cb2 = 0.0, cb3 = 0.0;
            if (arow) {
                const double *cr = p.cbound + (row0 + a) * CB_STRIDE;
                ra0 = __ldg(cr);
                ra2 = __ldg(cr + 2);
                ra3 = __ldg(cr + 3);
            }
#pragma unroll
            for (int h = 0; h < EPI_COLS / 32; ++h) {
                const long bcol = b0 + lane + 32 * h;
                if (bcol < n) {
                    const double *cc = p.cbound + (row0 + bcol) * CB_STRIDE;
                    cb1 = fmax(cb1, __ldg(cc + 1));
                    cb2 = fmax(cb2, __ldg(cc + 2));
                    cb3 = fmax(cb3, __ldg(cc + 3));
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                ra0 = fmax(ra0, __shfl_xor_sync(0xffffffffu, ra0, o));
                ra2 = fmax(ra2, __shfl_xor_sync(0xffffffffu, ra2, o));
                ra3 = fmax(ra3, __shfl_xor_sync(0xffffffffu, ra3, o));
                cb1 = fmax(cb1, __shfl_xor_sync(0xffffffffu, cb1, o));
                cb2 = fmax(cb2, __shfl_xor_sync(0xffffffffu, cb2, o));
                cb3 = fmax(cb3, __shfl_xor_sync(0xffffffffu, cb3, o));
            }
            const bool need_corr = !(ra0 * cb1 + ra2 * cb3 + ra3 * cb2 <= p.corr_floor);
            constexpr int FC = 8;  // columns per final-phase chunk
            // The final phase runs once per tile: a rolled loop keeps its code
            // small enough to stay in the instruction cache beside the
            // per-modulus code, so the register-resident last group is first
            // copied to a (cached) local array that the loop can index.
            uint32_t pk_l[EPI_COLS];
#pragma unroll
            for (int c = 0; c < EPI_COLS; ++c) pk_l[c] = pk[c];
#pragma unroll 1
            for (int c = 0; c < EPI_COLS / FC; ++c) {
                uint32_t w0[FC], w1[FC], w2[FC];
                if (PARKED >= 1) tmem_ld8(tmem + lane_off + 256u + col0 + (uint32_t)(c * FC), w0);
                if (PARKED >= 2) tmem_ld8(tmem + lane_off + 384u + col0 + (uint32_t)(c * FC), w1);
#pragma unroll
                for (int j = 0; j < FC; ++j) w2[j] = pk_l[c * FC + j];
                tmem_wait_ld();
                double xs[FC];
#pragma unroll
                for (int j = 0; j < FC; ++j) {
                    double yh = 0.0, yl = 0.0;
#pragma unroll
                    for (int dg = 0; dg < NDIG; ++dg) {
                        const int md = 2 * dg;              // first modulus of the digit
                        const int grp = md >> 2;
                        const uint32_t word = grp == LASTG ? w2[j] : (grp == 0 ? w0[j] : w1[j]);
                        const uint32_t dv = (word >> (16 * ((md >> 1) & 1))) & 0xffffu;
                        // exact int -> double: (2^52 + dv) - 2^52
                        const double r = __hiloint2double(0x43300000, (int)dv) - 4503599627370496.0;
                        yh = fma(r, p.f_hi[dg], yh);
                        yl = fma(r, p.f_lo[dg], yl);
                    }
                    const long b = b0 + c * FC + j;
                    const double rs_b = b < n ? __ldg(p.rowscale + row0 + b) : 0.0;
                    xs[j] = ((yh - rint(yh)) * p.M + yl * p.M) * (rs_a * rs_b);
                }
                if (need_corr && arow) {  // warp-uniform except for the row guard
                    for (int j = 0; j < FC; ++j) {
                        const long b = b0 + c * FC + j;
                        if (b < n) {
                            const double *rb = p.right + (row0 + b) * p.cwp;
                            double corr = 0.0;
                            for (int i = 0; i < p.cw; ++i) corr = fma(__ldg(la + i), __ldg(rb + i), corr);
                            xs[j] += corr;
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < FC; ++j) {
                    const long b = b0 + c * FC + j;
                    const bool valid = arow && b < n;
                    const double v = valid ? xs[j] : 0.0;
                    if (valid) {
                        if (!isfinite(v)) atomicExch(status, (int)RKB_ENONFINITE);
                        if (mirror) R[b * n + a] = v;  // lanes hold consecutive a: coalesced
                    }
                    stg[lane * STG_LD + j] = v;
                }
                {
                    // direct tile row segments of 8 columns through shared memory (coalesced rows)
                    __syncwarp();
                    const long a0 = (long)ti * BM + quarter * 32;
                    const long bc = b0 + c * FC;
#pragma unroll 4
                    for (int rr = 0; rr < 32; rr += 4) {
                        const int row = rr + (lane >> 3), col = lane & 7;
                        const long aa = a0 + row, bb = bc + col;
                        if (aa < n && bb < n) R[aa * n + bb] = stg[row * STG_LD + col];
                    }
                    __syncwarp();
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
    }
}

// ------------------------------------------------------------- host helpers
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)f;
    }
    return fn;
}

static int make_map(CUtensorMap *map, const void *ptr, long kpad, long rows) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) {
        set_error("cuTensorMapEncodeTiled is unavailable from the CUDA driver");
        return RKB_EUNSUPPORTED;
    }
    cuuint64_t dims[2] = {(cuuint64_t)kpad, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kpad};
    cuuint32_t box[2] = {(cuuint32_t)BKB, (cuuint32_t)BM};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(ptr), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d) for a %ld x %ld residue matrix", (int)r, rows, kpad);
        return RKB_EINVAL;
    }
    return RKB_OK;
}

}  // namespace split
}  // namespace rkb

using namespace rkb;
using namespace rkb::split;

extern "C" int rkb_split_rows(const double *d_Pv, const double *d_Qv, long orb_ld, const long *d_pairs,
                              const long *d_row_pair, const int *d_row_k, long nrows, const double *d_w, int nv,
                              int ng, const double *d_ktab, const long *d_koff, int bits, int n_mod,
                              const int *moduli, signed char *d_resA, signed char *d_resB, long kpad,
                              long row_base, long nrows_total, double *d_rowscale, double *d_left,
                              double *d_right, double *d_cbound, int cwp, double *d_xwork,
                              const int *d_zcount, void *stream) {
    RKB_CHECK_ARG(nv >= 2 && ng >= 1 && ng <= RKB_MAX_NG, "invalid grid (nv=%d, ng=%d)", nv, ng);
    RKB_CHECK_ARG(bits >= 8 && bits <= 50, "bits must be in [8, 50] (got %d)", bits);
    RKB_CHECK_ARG(n_mod >= 1 && n_mod <= MAXMOD, "1..%d moduli supported (got %d)", MAXMOD, n_mod);
    RKB_CHECK_ARG(kpad % BKB == 0 && kpad >= (long)(nv - 1) * ng, "kpad must be a multiple of %d >= body width",
                  BKB);
    RKB_CHECK_ARG(cwp >= ng + 2, "correction width must be >= ng + 2");
    RKB_CHECK_ARG(d_cbound != nullptr, "the correction-bound array is required");
    RKB_CHECK_ARG(row_base >= 0 && row_base + nrows <= nrows_total, "row range outside the residue matrices");
    if (nrows == 0) return RKB_OK;
    RowsArgs a;
    a.P = d_Pv; a.Q = d_Qv; a.orb_ld = orb_ld; a.pairs = d_pairs; a.row_pair = d_row_pair; a.row_k = d_row_k;
    a.nrows = nrows; a.w = d_w; a.nv = nv; a.ng = ng; a.ktab = d_ktab; a.koff = d_koff; a.bits = bits;
    a.n_mod = n_mod;
    for (int i = 0; i < MAXMOD; ++i) {
        const int m = i < n_mod ? moduli[i] : 256;
        RKB_CHECK_ARG(m >= 2 && m <= 256, "moduli must lie in [2, 256]");
        a.mod[i] = m;
        a.magic[i] = (uint32_t)((1ULL << 32) / (unsigned long long)m + 1ULL);
        a.c20[i] = (uint32_t)((1u << 20) % (uint32_t)m);
        a.bias[i] = (uint32_t)m << 20;  // hi + bias >= 0 for |hi| <= 2^20
        a.inv_mod[i] = 1.0 / (double)m;
    }
    a.resA = d_resA; a.resB = d_resB; a.kpad = kpad; a.row_base = row_base; a.nrows_total = nrows_total;
    a.rowscale = d_rowscale; a.left = d_left; a.right = d_right; a.cbound = d_cbound; a.cwp = cwp;
    a.xwork = d_xwork;
    RKB_CHECK_ARG(d_xwork != nullptr && d_zcount != nullptr, "the row workspace and Z counts are required");
    RKB_CHECK_ARG(bits <= 40, "the residue path handles |x| <= 2^40 (bits <= 40)");
    RKB_CHECK_ARG(kpad % 16 == 0, "kpad must be a multiple of 16");
    const long np = ((long)nv * ng + 1) & ~1L, nvp = ((long)nv + 1) & ~1L;
    const size_t per_warp = (size_t)(np + nvp) * sizeof(double);
    const int warps = 4;
    size_t smem = (size_t)warps * per_warp;
    RKB_CHECK_ARG(smem <= 200 * 1024, "grid too large for the split row kernel");
    dim3 grid((unsigned)ceil_div(nrows, warps)), block(32 * warps);
    cudaStream_t st = as_stream(stream);
    RKB_CHECK_ARG(((uintptr_t)d_resA % 16) == 0 && (d_resB == nullptr || ((uintptr_t)d_resB % 16) == 0),
                  "residue buffers must be 16-byte aligned");
#define RKB_SR_CASE(NGV)                                                                              \
    case NGV: {                                                                                       \
        RKB_CUDA(set_smem(split_rows_kernel<NGV>, (int)smem));                                         \
        split_rows_kernel<NGV><<<grid, block, smem, st>>>(a);                                         \
        break;                                                                                        \
    }
    switch (ng) {
        RKB_SR_CASE(5) RKB_SR_CASE(7) RKB_SR_CASE(8) RKB_SR_CASE(9) RKB_SR_CASE(11)
        default: {
            RKB_CUDA(set_smem(split_rows_kernel<0>, (int)smem));
            split_rows_kernel<0><<<grid, block, smem, st>>>(a);
        }
    }
#undef RKB_SR_CASE
    RKB_LAUNCHED("split_rows_kernel");
    const long nthreads = nrows * (kpad / 16);
    split_residues_kernel<<<(unsigned)ceil_div(nthreads, 256), 256, 0, st>>>(a, d_zcount);
    RKB_LAUNCHED("split_residues_kernel");
    return RKB_OK;
}

extern "C" int rkb_split_rows_cells(const double *d_Pv, const double *d_Qv, long orb_ld, const long *d_pairs,
                                    const long *d_row_pair, const int *d_row_k, long nrows, const double *d_w,
                                    int nv, int ng, const double *d_ktab, const long *d_koff,
                                    const double *d_ktab_t, const long *d_koff_t, int max_z, int bits,
                                    int n_mod, const int *moduli, signed char *d_resA, signed char *d_resB,
                                    long kpad, long row_base, long nrows_total, double *d_rowscale, double *d_left,
                                    double *d_right, double *d_cbound, int cwp, void *stream) {
    RKB_CHECK_ARG(nv >= 2 && ng >= 5 && ng <= 11, "the cell row kernel takes 5 <= ng <= 11 (got %d)", ng);
    RKB_CHECK_ARG(max_z >= 0 && max_z <= CELL_ZMAX, "the cell row kernel takes <= %d Z columns (got %d)", CELL_ZMAX,
                  max_z);
    const long threads = ((long)nv + max_z + 31) / 32 * 32;
    RKB_CHECK_ARG(threads <= 256, "grid too long for the cell row kernel (%d cells + %d Z columns > 256)", nv,
                  max_z);
    RKB_CHECK_ARG(bits >= 8 && bits <= 40, "bits must be in [8, 40] (got %d)", bits);
    RKB_CHECK_ARG(n_mod >= 1 && n_mod <= MAXMOD, "1..%d moduli supported (got %d)", MAXMOD, n_mod);
    RKB_CHECK_ARG(kpad % BKB == 0 && kpad >= (long)(nv - 1) * ng + max_z, "kpad must be a multiple of %d >= %ld",
                  BKB, (long)(nv - 1) * ng + max_z);
    RKB_CHECK_ARG(cwp >= ng + 2, "correction width must be >= ng + 2");
    RKB_CHECK_ARG(d_cbound != nullptr, "the correction-bound array is required");
    RKB_CHECK_ARG(row_base >= 0 && row_base + nrows <= nrows_total, "row range outside the residue matrices");
    RKB_CHECK_ARG(((uintptr_t)d_resA % 16) == 0 && (d_resB == nullptr || ((uintptr_t)d_resB % 16) == 0),
                  "residue buffers must be 16-byte aligned");
    if (nrows == 0) return RKB_OK;
    RowsArgs a = {};
    a.P = d_Pv; a.Q = d_Qv; a.orb_ld = orb_ld; a.pairs = d_pairs; a.row_pair = d_row_pair; a.row_k = d_row_k;
    a.nrows = nrows; a.w = d_w; a.nv = nv; a.ng = ng; a.ktab = d_ktab; a.koff = d_koff; a.bits = bits;
    a.n_mod = n_mod;
    for (int i = 0; i < MAXMOD; ++i) {
        const int m = i < n_mod ? moduli[i] : 256;
        RKB_CHECK_ARG(m >= 2 && m <= 256, "moduli must lie in [2, 256]");
        a.mod[i] = m;
        a.inv_mod[i] = 1.0 / (double)m;
    }
    a.resA = d_resA; a.resB = d_resB; a.kpad = kpad; a.row_base = row_base; a.nrows_total = nrows_total;
    a.rowscale = d_rowscale; a.left = d_left; a.right = d_right; a.cbound = d_cbound; a.cwp = cwp;
    RKB_CHECK_ARG(d_ktab_t != nullptr && d_koff_t != nullptr, "the cell-minor factor tables are required");
    const size_t smem = ((((size_t)nv * (ng | 1) + 64 + 1) & ~(size_t)1) * sizeof(double)) + (size_t)n_mod * (kpad + CELL_ZMAX);
    RKB_CHECK_ARG(smem <= 200 * 1024, "row images too large for shared memory");
    cudaStream_t st = as_stream(stream);
    const dim3 grid((unsigned)nrows), block((unsigned)threads);
#define RKB_CELL_CASE(NGV)                                                         \
    case NGV:                                                                      \
        RKB_CUDA(set_smem(split_rows_cell_kernel<NGV>, (int)smem));                \
        split_rows_cell_kernel<NGV><<<grid, block, smem, st>>>(a, d_ktab_t, d_koff_t); \
        break;
    switch (ng) {
        RKB_CELL_CASE(5) RKB_CELL_CASE(6) RKB_CELL_CASE(7) RKB_CELL_CASE(8) RKB_CELL_CASE(9) RKB_CELL_CASE(10)
        default:
            RKB_CELL_CASE(11)
    }
#undef RKB_CELL_CASE
    RKB_LAUNCHED("split_rows_cell_kernel");
    return RKB_OK;
}

extern "C" long rkb_split_fused_body_width(int nv, int ng) {
    if (nv < 2 || ng < 1 || ng > 32) return -1;
    return rkb::split::fused_body_width(nv, ng);
}

extern "C" int rkb_split_rows_fused(const double *d_Pv, const double *d_Qv, long orb_ld, const long *d_pairs,
                                    const long *d_row_pair, const int *d_row_k, long nrows, const double *d_w,
                                    int nv, int ng, const double *d_ktab, const long *d_koff, int max_z, int bits,
                                    int n_mod, const int *moduli, signed char *d_resA, signed char *d_resB,
                                    long kpad, long row_base, long nrows_total, double *d_rowscale, double *d_left,
                                    double *d_right, double *d_cbound, int cwp, void *stream) {
    RKB_CHECK_ARG(nv >= 2 && ng >= 5 && ng <= 11, "the fused row kernel takes 5 <= ng <= 11 (got %d)", ng);
    RKB_CHECK_ARG(fused_passes(nv, ng) <= FUSED_PMAX, "grid too long for the fused row kernel (%ld passes > %d)",
                  fused_passes(nv, ng), FUSED_PMAX);
    RKB_CHECK_ARG(max_z >= 0 && max_z <= FUSED_ZMAX, "the fused row kernel takes <= %d Z columns (got %d)",
                  FUSED_ZMAX, max_z);
    RKB_CHECK_ARG(bits >= 8 && bits <= 40, "bits must be in [8, 40] (got %d)", bits);
    RKB_CHECK_ARG(n_mod >= 1 && n_mod <= MAXMOD, "1..%d moduli supported (got %d)", MAXMOD, n_mod);
    RKB_CHECK_ARG(kpad % BKB == 0 && kpad >= fused_body_width(nv, ng) + max_z,
                  "kpad must be a multiple of %d >= %ld", BKB, fused_body_width(nv, ng) + max_z);
    RKB_CHECK_ARG(cwp >= ng + 2 && cwp <= 32, "correction width must be in [ng + 2, 32]");
    RKB_CHECK_ARG(d_cbound != nullptr, "the correction-bound array is required");
    RKB_CHECK_ARG(row_base >= 0 && row_base + nrows <= nrows_total, "row range outside the residue matrices");
    RKB_CHECK_ARG(((uintptr_t)d_resA % 16) == 0 && (d_resB == nullptr || ((uintptr_t)d_resB % 16) == 0),
                  "residue buffers must be 16-byte aligned");
    if (nrows == 0) return RKB_OK;
    RowsArgs a = {};
    a.P = d_Pv; a.Q = d_Qv; a.orb_ld = orb_ld; a.pairs = d_pairs; a.row_pair = d_row_pair; a.row_k = d_row_k;
    a.nrows = nrows; a.w = d_w; a.nv = nv; a.ng = ng; a.ktab = d_ktab; a.koff = d_koff; a.bits = bits;
    a.n_mod = n_mod;
    for (int i = 0; i < MAXMOD; ++i) {
        const int m = i < n_mod ? moduli[i] : 256;
        RKB_CHECK_ARG(m >= 2 && m <= 256, "moduli must lie in [2, 256]");
        a.mod[i] = m;
        a.inv_mod[i] = 1.0 / (double)m;
    }
    a.resA = d_resA; a.resB = d_resB; a.kpad = kpad; a.row_base = row_base; a.nrows_total = nrows_total;
    a.rowscale = d_rowscale; a.left = d_left; a.right = d_right; a.cbound = d_cbound; a.cwp = cwp;
    const int warps = 4;
    dim3 grid((unsigned)ceil_div(nrows, warps)), block(32 * warps);
    cudaStream_t st = as_stream(stream);
    switch (ng) {
        case 5: split_rows_fused_kernel<5><<<grid, block, 0, st>>>(a); break;
        case 6: split_rows_fused_kernel<6><<<grid, block, 0, st>>>(a); break;
        case 7: split_rows_fused_kernel<7><<<grid, block, 0, st>>>(a); break;
        case 8: split_rows_fused_kernel<8><<<grid, block, 0, st>>>(a); break;
        case 9: split_rows_fused_kernel<9><<<grid, block, 0, st>>>(a); break;
        case 10: split_rows_fused_kernel<10><<<grid, block, 0, st>>>(a); break;
        default: split_rows_fused_kernel<11><<<grid, block, 0, st>>>(a); break;
    }
    RKB_LAUNCHED("split_rows_fused_kernel");
    return RKB_OK;
}

extern "C" int rkb_split_contract(const signed char *d_resA, const signed char *d_resB, long kpad,
                                  long nrows_total, int n_mod, const int *moduli, const int *pair_inv,
                                  const double *f_hi,
                                  const double *f_lo, double M, const double *d_rowscale, const double *d_left,
                                  const double *d_right, const double *d_cbound, double corr_floor, int cw,
                                  int cwp, const long *d_grp_row0,
                                  const long *d_grp_n, const long *d_grp_kdim, const long *d_grp_out,
                                  const int *d_tasks, long n_tasks, double *d_out, int *d_status, void *stream) {
    RKB_CHECK_ARG(n_mod >= 1 && n_mod <= MAXMOD, "1..%d moduli supported (got %d)", MAXMOD, n_mod);
    RKB_CHECK_ARG(kpad % BKB == 0 && kpad > 0 && kpad <= 3456, "kpad must be a positive multiple of %d, <= 3456",
                  BKB);
    RKB_CHECK_ARG((long)n_mod * nrows_total < (1L << 31), "residue matrices too tall for 32-bit TMA rows");
    RKB_CHECK_ARG(d_status != nullptr, "a device status word is required");
    RKB_CHECK_ARG(cw <= cwp, "cw must be <= cwp");
    RKB_CHECK_ARG(d_cbound != nullptr && corr_floor >= 0.0, "correction bounds and a nonnegative floor are required");
    if (n_tasks == 0) return RKB_OK;
    CUtensorMap mA, mB;
    int rc = make_map(&mA, d_resA, kpad, (long)n_mod * nrows_total);
    if (rc) return rc;
    rc = make_map(&mB, d_resB ? d_resB : d_resA, kpad, (long)n_mod * nrows_total);
    if (rc) return rc;
    CrtArgs p;
    p.rowscale = d_rowscale; p.left = d_left; p.right = d_right; p.cbound = d_cbound; p.corr_floor = corr_floor;
    p.cwp = cwp; p.cw = cw;
    p.grp_row0 = d_grp_row0; p.grp_n = d_grp_n; p.grp_kdim = d_grp_kdim; p.grp_out = d_grp_out;
    p.tasks = d_tasks; p.n_tasks = n_tasks; p.nrows_total = nrows_total; p.out = d_out; p.status = d_status;
    p.n_mod = n_mod; p.M = M;
    const int ndig = (n_mod + 1) / 2;
    for (int i = 0; i < MAXMOD; ++i) {
        const int m = i < n_mod ? moduli[i] : 256;
        RKB_CHECK_ARG(m >= 2 && m <= 256, "moduli must lie in [2, 256]");
        p.mod[i] = m;
        p.magic[i] = (uint32_t)((1ULL << 32) / (unsigned long long)m + 1ULL);
        p.bias[i] = (uint32_t)m << 18;
        p.f_hi[i] = i < ndig ? f_hi[i] : 0.0;
        p.f_lo[i] = i < ndig ? f_lo[i] : 0.0;
    }
    for (int i = 0; i < MAXMOD / 2; ++i) p.pinv[i] = i < n_mod / 2 ? (uint32_t)pair_inv[i] : 1u;
    long grid = n_tasks < sm_count() ? n_tasks : sm_count();
    cudaStream_t st = as_stream(stream);
#define RKB_CRT_CASE(NM)                                                                                     \
    case NM: {                                                                                               \
        RKB_CUDA(set_smem(crt_syrk_kernel<NM>, (int)SMEM_BYTES));                                            \
        crt_syrk_kernel<NM><<<(unsigned)grid, THREADS, SMEM_BYTES, st>>>(mA, mB, p);                         \
        break;                                                                                               \
    }
    switch (n_mod) {
        RKB_CRT_CASE(4) RKB_CRT_CASE(5) RKB_CRT_CASE(6) RKB_CRT_CASE(7) RKB_CRT_CASE(8) RKB_CRT_CASE(9)
        RKB_CRT_CASE(10) RKB_CRT_CASE(11) RKB_CRT_CASE(12)
        default:
            set_error("split contraction compiled for 4..12 moduli (got %d)", n_mod);
            return RKB_EINVAL;
    }
#undef RKB_CRT_CASE
    RKB_LAUNCHED("crt_syrk_kernel");
    return RKB_OK;
}

// ---------------------------------------------------------------------------
// Certificate of each (ion, k) table from the row records, before or after the
// contraction.  Rounding row a to the quantum h_a = 2^(e_a - bits) moves entry
// (a, b) by about h_a |[X|Z]_b| + h_b |[X|Z]_a| (a random walk of K rounding
// errors against the other row), so the Schwarz-relative error of the table
// is estimated by
//     est = max_a h_a / sqrt|R_aa|  *  max_b |[X|Z]_b| / sqrt|R_bb|
// (rows with [X|Z] = 0 carry no rounding and are skipped; a vanishing or
// non-finite diagonal gives est = inf).  Tables with est > limit are counted in
// *flagged; the host recomputes them in FP64.  One 1024-thread block per table.
namespace rkb {
namespace split {
constexpr int CERT_THREADS = 1024;

__global__ void __launch_bounds__(CERT_THREADS) certify_kernel(const long *__restrict__ grp_row0,
                                                      const long *__restrict__ grp_n,
                                                      const double *__restrict__ rowscale,
                                                      const double *__restrict__ cbound, double limit,
                                                      double *__restrict__ est, int *__restrict__ flagged) {
    __shared__ double sm1[CERT_THREADS / 32], sm2[CERT_THREADS / 32];
    __shared__ int sbad[CERT_THREADS / 32];
    const long g = blockIdx.x;
    const long row0 = grp_row0[g], n = grp_n[g];
    double m1 = 0.0, m2 = 0.0;
    bool bad = false;
    for (long i = threadIdx.x; i < n; i += blockDim.x) {
        const long r = row0 + i;
        const double nrm = cbound[r * CB_STRIDE + 4];
        if (nrm == 0.0) continue;
        const double rd = sqrt(fabs(cbound[r * CB_STRIDE + 5]));
        const double t1 = rowscale[r] / rd, t2 = nrm / rd;
        if (!(t1 <= DBL_MAX) || !(t2 <= DBL_MAX)) {
            bad = true;
        } else {
            m1 = fmax(m1, t1);
            m2 = fmax(m2, t2);
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    const int badw = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
        sm1[wid] = m1;
        sm2[wid] = m2;
        sbad[wid] = badw;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        bool any = false;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            m1 = fmax(m1, sm1[w]);
            m2 = fmax(m2, sm2[w]);
            any |= sbad[w] != 0;
        }
        const double e = any ? INFINITY : m1 * m2;
        est[g] = e;
        if (!(e <= limit)) atomicAdd(flagged, 1);
    }
}
}  // namespace split
}  // namespace rkb

extern "C" int rkb_split_certify(const long *d_grp_row0, const long *d_grp_n, long n_groups, const double *d_rowscale,
                                 const double *d_cbound, double limit, double *d_est, int *d_flagged, void *stream) {
    RKB_CHECK_ARG(n_groups >= 0 && n_groups <= 0x7fffffffL, "invalid group count %ld", n_groups);
    RKB_CHECK_ARG(limit >= 0.0, "the certificate limit must be >= 0");
    RKB_CHECK_ARG(d_flagged != nullptr && (n_groups == 0 || (d_grp_row0 && d_grp_n && d_rowscale && d_cbound && d_est)),
                  "null argument");
    cudaStream_t st = as_stream(stream);
    RKB_CUDA(cudaMemsetAsync(d_flagged, 0, sizeof(int), st));
    if (n_groups == 0) return RKB_OK;
    certify_kernel<<<(unsigned)n_groups, CERT_THREADS, 0, st>>>(d_grp_row0, d_grp_n, d_rowscale, d_cbound, limit,
                                                               d_est, d_flagged);
    RKB_LAUNCHED("certify_kernel");
    return RKB_OK;
}

// ---------------------------------------------------------------------------
// rkb_split_rows_noalloc: rkb_split_rows whose row workspace is a fixed array
// compiled into this library instead of caller memory.  It is meant for hosts
// that cannot call cudaMalloc on this path: a C or Fortran program that links
// only this ABI and hands over buffers from its own pool, or a process that
// plans every device allocation up front and may not have cudaMalloc /
// cudaFree synchronise the device in the middle of its pipelined streams.
//
// The array holds RKB_SPLIT_ROWS_NOALLOC_MAX_DOUBLES doubles (16 MiB) on every
// GPU that loads the library, until the process exits.  The host name of a
// __device__ array is only a host-side stand-in, so its device address is
// looked up per device with cudaGetSymbolAddress, on the first call made with
// that device current; make that first call before any stream capture.
// Every call shares the one array, so calls that overlap on the GPU (other
// streams, other host threads) race and must be serialised by the caller.
// Nothing needs clearing between calls: the row kernel writes every element
// of each row [X | Z | 0] that the residue kernel later reads.
namespace rkb {
namespace split {
static __device__ __align__(256) double g_noalloc_xwork[RKB_SPLIT_ROWS_NOALLOC_MAX_DOUBLES];

constexpr int NOALLOC_MAX_DEVICES = 64;
static double *g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};
static std::mutex g_noalloc_mutex;
}  // namespace split
}  // namespace rkb

extern "C" int rkb_split_rows_noalloc(const double *d_Pv, const double *d_Qv, long orb_ld, const long *d_pairs,
                                      const long *d_row_pair, const int *d_row_k, long nrows, const double *d_w,
                                      int nv, int ng, const double *d_ktab, const long *d_koff, int bits,
                                      int n_mod, const int *moduli, signed char *d_resA, signed char *d_resB,
                                      long kpad, long row_base, long nrows_total, double *d_rowscale,
                                      double *d_left, double *d_right, double *d_cbound, int cwp,
                                      const int *d_zcount, void *stream) {
    const long cap = (long)RKB_SPLIT_ROWS_NOALLOC_MAX_DOUBLES;
    RKB_CHECK_ARG(kpad > 0 && nrows >= 0 && row_base >= 0, "invalid row range or width");
    RKB_CHECK_ARG(row_base <= cap / kpad && nrows <= cap / kpad - row_base,
                  "rows [0, %ld) of width %ld need %ld workspace doubles; the fixed workspace holds %ld "
                  "(use rkb_split_rows with a caller buffer)",
                  row_base + nrows, kpad, (row_base + nrows) * kpad, cap);
    int dev = -1;
    RKB_CUDA(cudaGetDevice(&dev));
    RKB_CHECK_ARG(dev >= 0 && dev < NOALLOC_MAX_DEVICES, "device ordinal %d out of range", dev);
    double *ws = nullptr;
    {
        std::lock_guard<std::mutex> guard(g_noalloc_mutex);
        if (g_noalloc_addr[dev] == nullptr) {
            void *addr = nullptr;
            RKB_CUDA(cudaGetSymbolAddress(&addr, g_noalloc_xwork));
            g_noalloc_addr[dev] = static_cast<double *>(addr);
        }
        ws = g_noalloc_addr[dev];
    }
    return rkb_split_rows(d_Pv, d_Qv, orb_ld, d_pairs, d_row_pair, d_row_k, nrows, d_w, nv, ng, d_ktab, d_koff,
                          bits, n_mod, moduli, d_resA, d_resB, kpad, row_base, nrows_total, d_rowscale, d_left,
                          d_right, d_cbound, cwp, ws, d_zcount, stream);
}
