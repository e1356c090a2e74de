"""Host planning for the split-precision (Ozaki-II / CRT) R^k engine.

Factored Green operator
-----------------------
With g = w*rho on the cell Gauss grid, atomx's R^k(ac;bd) = g_ac^T G g_bd
(numerics/yk.py:88-154 builds Y = G g; numerics/bspline/slater.py:130
contracts it).  G is symmetric: its off-cell blocks are the exact kernel
samples r_<^k / r_>^{k+1}, and inside a cell the interpolatory partial
matrices satisfy mo + mo^T = 1, so G_ij = u_i v_j mo_ij + v_i u_j mo_ji with
u = r^-(k+1), v = r^k.  Off-diagonal cell blocks are rank one, so G is
block-semiseparable.

Split G at cell 0 (the cell [0, r_min] whose partial rule acts on an
endpoint-singular integrand and whose block is violently indefinite) and keep
the core in FP64:

  R = X_ac . X_bd - Z_ac . Z_bd + left_ac . right_bd

* body (cells >= 1): a block Cholesky of the semiseparable G_bb computed by
  the recursion  S_m = D_m - sigma_m u_m u_m^T,  L_mm L_mm^T = S_m + Delta_m,
  c_m = L_mm^{-1} (v_m - sigma_m u_m),  sigma_{m+1} = sigma_m + |c_m|^2,
  which gives X = L^T g_b per row in O(N ng):
      X_m = L_mm^T g_m + c_m * sum_{m' > m} u_m'.g_m'.
  Delta_m (a modified-Cholesky shift, rank = number of Schur eigenvalues
  below tau * lambda_max of the diagonally scaled block) is returned as
  extra columns Z with a negative sign: g^T Delta g = sum_e (z_e . g_m)^2;
* core (cell 0) and the core-body coupling G_cb = v_0 u_b^T stay in FP64:
      left  = [g_0, alpha sx, q / sx],   right = [G_00 g_0, q / sx, alpha sx]
  with alpha = v_0 . g_0 (the core multipole moment), q = u_b . g_b (the
  body's potential moment at the origin), so left_ac . right_bd =
  g0_ac^T G_00 g0_bd + alpha_ac q_bd + q_ac alpha_bd.  The scale
  sx = r_b^-(k+1)/2 r_l^-k/2 (r_l the last core node, r_b the first body
  node) bounds both |alpha sx| and |q / sx| by |g|_1 / sqrt(r_b).

Folding the coupling into X instead (X += ell alpha with ell = L^-1 u_b, the
core Schur complement G_00 - |ell|^2 v_0 v_0^T left in FP64) is exact in
real arithmetic but |ell|^2 ~ r_b^-(2k+1): on coarse grids (first body node
near 1e-5, cell ratios ~60) the folded term exceeds R by up to 1e20 and
cancels against the Schur complement, which no fixed-point split survives.
Kept apart, alpha_ac q_bd is as small as the physics makes it.

|X_ac.X_bd| <= |X_ac||X_bd| = sqrt(R_acac R_bdbd) (up to the small Delta and
the core terms), so a per-row fixed-point split of X has an error bounded
relative to the Schwarz scale of every entry, which is what the split engine
needs.  Where the core block itself cancels most of the body energy (wide
origin cells at mid k: g0^T G_00 g0 near -R_body), |X|^2 exceeds R_acac by
the same factor and the split's error grows with it; the engines certify
every multipole table from per-row norms and recompute the ones that fail in
FP64.

CRT constants
-------------
Pairwise-coprime moduli m_i <= 256 (int8 residues in [-128, 127]), M = prod m_i.
The device reduces each int32 accumulator to r_i in [0, m_i) and merges the
residues of consecutive moduli into one digit d_p = r_2p + m_2p t,
t = (r_2p+1 - r_2p) m_2p^-1 mod m_2p+1, a residue mod D_p = m_2p m_2p+1
(< 2^16); an odd last modulus stays a digit of its own.  An integer x with
|x| < M/2 is rebuilt from the digits as x = M * frac(sum_p d_p f_p),
f_p = (M/D_p) [(M/D_p)^-1 mod D_p] / M mod 1.  f_p is split into f_hi (a
multiple of 2^-34) and f_lo = f_p - f_hi, so sum d_p f_hi is exact in one
double for up to 6 digits below 2^16.
"""
from __future__ import annotations

import math
from fractions import Fraction
from functools import lru_cache

import numpy as np

from .yk import yk_partial_matrices

__all__ = ["MODULI", "bits_for_moduli", "crt_constants", "digit_moduli", "moduli_needed", "green_factor",
           "green_factor_packed", "pack_factors", "concat_tables", "table_z_count", "factor_table_layout"]

#: Pairwise-coprime moduli, largest first (256 = 2^8; 255 = 3*5*17; 253 = 11*23;
#: 247 = 13*19; 217 = 7*31; the rest are primes).
MODULI = (256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217)
MAX_MODULI = 12


def moduli_needed(bits: int, kdim: int) -> int:
    """Fewest leading moduli whose product exceeds 2 * kdim * 2^(2*bits) + 2."""
    need = 2 * kdim * (1 << (2 * bits)) + 2
    prod = 1
    for i, m in enumerate(MODULI):
        prod *= m
        if prod > need:
            return i + 1
    raise ValueError(f"{bits}-bit splits of length {kdim} need more than {MAX_MODULI} int8 moduli")


def bits_for_moduli(n_mod: int, kdim: int, cap: int = 40) -> int:
    """Widest split (bits, at most ``cap``) whose products the first n_mod moduli
    still hold exactly: the largest b with 2 * kdim * 2^(2b) + 2 < prod m_i."""
    M = math.prod(MODULI[:n_mod])
    b = 0
    while b < cap and 2 * kdim * (1 << (2 * (b + 1))) + 2 < M:
        b += 1
    return b


def digit_moduli(n_mod: int) -> list[int]:
    """Moduli of the merged digits: m_0 m_1, m_2 m_3, ... (+ the odd last one)."""
    ms = MODULI[:n_mod]
    out = [ms[i] * ms[i + 1] for i in range(0, n_mod - 1, 2)]
    if n_mod % 2:
        out.append(ms[-1])
    return out


@lru_cache(maxsize=16)
def crt_constants(n_mod: int):
    """(moduli, f_hi, f_lo, M as double, pair inverses) for the first n_mod moduli.

    f_hi / f_lo are per merged digit (see the module docstring); pair_inv[p] is
    m_2p^-1 mod m_2p+1.
    """
    if not 1 <= n_mod <= MAX_MODULI:
        raise ValueError("1..12 moduli supported")
    ms = MODULI[:n_mod]
    M = math.prod(ms)
    f_hi, f_lo = [], []
    for D in digit_moduli(n_mod):
        Mi = M // D
        inv = pow(Mi % D, -1, D)
        f = Fraction((Mi * inv) % M, M)
        hi = Fraction(round(f * (1 << 34)), 1 << 34)
        f_hi.append(float(hi))          # exact: a multiple of 2^-34 below 1
        f_lo.append(float(f - hi))
    pair_inv = [pow(ms[i], -1, ms[i + 1]) for i in range(0, n_mod - 1, 2)]
    return (np.asarray(ms, dtype=np.int32), np.asarray(f_hi), np.asarray(f_lo), float(M),
            np.asarray(pair_inv, dtype=np.int32))


def green_factor(r_flat: np.ndarray, ng: int, k: int, tau: float = 1e-3) -> dict:
    """Structured modified Cholesky of the body Green matrix (see module doc)."""
    r = np.asarray(r_flat, dtype=np.float64)
    nv = r.shape[0] // ng
    mo, mi = yk_partial_matrices(ng)
    u = (r ** (-(k + 1))).reshape(nv, ng)
    v = (r ** k).reshape(nv, ng)
    Lb = np.zeros((nv, ng, ng))
    C = np.zeros((nv, ng))
    zcell, zvec = [], []
    sigma = 0.0
    for m in range(1, nv):
        D = u[m][:, None] * v[m][None, :] * mo + v[m][:, None] * u[m][None, :] * mi
        D = 0.5 * (D + D.T)
        S = D - sigma * np.outer(u[m], u[m])
        d = np.sqrt(np.abs(np.diag(D)))
        lam, V = np.linalg.eigh(S / np.outer(d, d))
        floor = tau * lam[-1]
        for e in np.flatnonzero(lam < floor):
            shift = max(abs(lam[e]), floor) - lam[e]
            z = np.sqrt(shift) * V[:, e] * d
            zcell.append(m)
            zvec.append(z)
            S = S + np.outer(z, z)
        Lm = np.linalg.cholesky(S)
        Lb[m] = Lm
        C[m] = np.linalg.solve(Lm, v[m] - sigma * u[m])
        sigma += float(C[m] @ C[m])
    G00 = u[0][:, None] * v[0][None, :] * mo + v[0][:, None] * u[0][None, :] * mi
    sx = float(np.sqrt(u[1, 0]) / np.sqrt(v[0, -1]))
    return dict(k=k, nv=nv, ng=ng, u=u, v0=v[0].copy(), Lb=Lb, C=C, G00=G00, sx=sx,
                zcell=np.asarray(zcell, dtype=np.int64), zvec=np.asarray(zvec).reshape(-1, ng))


def green_factor_packed(r_flat: np.ndarray, ng: int, k: int, tau: float = 1e-3) -> np.ndarray:
    """The same factorisation as ``green_factor``, computed natively and
    returned packed (``pack_factors`` layout of one table)."""
    from . import _native
    L = _native.load()
    r = np.ascontiguousarray(r_flat, dtype=np.float64)
    nv = r.shape[0] // ng
    mo, mi = yk_partial_matrices(ng)
    mo = np.ascontiguousarray(mo, dtype=np.float64)
    mi = np.ascontiguousarray(mi, dtype=np.float64)
    cap = nv * ng + nv * ng * ng + nv * ng + ng + ng * ng + 2 + nv * ng * (ng + 1)
    out = np.empty(cap, dtype=np.float64)
    got = L.rkb_green_factor(r.ctypes.data, nv, ng, int(k), float(tau), mo.ctypes.data, mi.ctypes.data,
                             out.ctypes.data, cap)
    if got < 0:
        _native.check(int(-got), "rkb_green_factor")
    return out[:got].copy()


def table_z_count(table: np.ndarray, nv: int, ng: int) -> int:
    """Number of Z columns of one packed factor table."""
    return int(table[factor_table_layout(nv, ng)["nz"]])


def concat_tables(tables: list[np.ndarray]) -> tuple[np.ndarray, np.ndarray]:
    """Concatenate packed tables: (flat doubles, offsets by list index)."""
    offs = np.concatenate([[0], np.cumsum([t.shape[0] for t in tables])])[:-1].astype(np.int64)
    return np.concatenate(tables), offs


def factor_table_layout(nv: int, ng: int) -> dict:
    """Offsets (in doubles) of the pieces of one packed factor table."""
    n = nv * ng
    o = {"u": 0, "Lb": n}
    o["C"] = o["Lb"] + nv * ng * ng
    o["v0"] = o["C"] + nv * ng
    o["G00"] = o["v0"] + ng
    o["sx"] = o["G00"] + ng * ng
    o["nz"] = o["sx"] + 1
    o["z"] = o["nz"] + 1
    return o


def pack_factors(factors: list[dict]) -> tuple[np.ndarray, np.ndarray]:
    """Concatenate per-k factor tables: returns (flat doubles, offsets by list index).

    Layout of one table (doubles): u[N] | Lb[nv][ng][ng] | C[nv][ng] | v0[ng] |
    G00[ng][ng] | sx | nZ | nZ x (cell, z[ng]).
    """
    parts, offs, off = [], [], 0
    for F in factors:
        nz = F["zcell"].shape[0]
        z = np.concatenate([F["zcell"].astype(np.float64)[:, None], F["zvec"]], axis=1).ravel() if nz else \
            np.zeros(0)
        t = np.concatenate([F["u"].ravel(), F["Lb"].ravel(), F["C"].ravel(), F["v0"], F["G00"].ravel(),
                            [float(F["sx"]), float(nz)], z])
        offs.append(off)
        parts.append(t)
        off += t.shape[0]
    return np.concatenate(parts), np.asarray(offs, dtype=np.int64)
