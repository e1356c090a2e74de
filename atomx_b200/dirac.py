"""Dirac-Coulomb spinor generator for the synthetic R^k workloads (host only).

The engine's inputs are B-spline coefficient vectors (P, Q) of relativistic
spinor orbitals.  The workloads use the lowest positive-energy eigenvectors of
the Dirac-Coulomb Hamiltonian in a kinetically balanced B-spline basis, as
atomx builds them in ``build_dirac_matrices`` / ``solve_dirac``
(atomx numerics/bspline/dirac_assembly.py:82-155 and :471-611):

* Galerkin blocks on the cell Gauss grid: overlap and -Z/r on each component,
  H_QQ shifted by -2c^2 S_QQ, and the two P-Q couplings
  H_PQ = -c <P|dQ/dr> + kappa c <P|Q/r>, H_QP = c <Q|dP/dr> + kappa c <Q|P/r>;
* the Bloch boundary correction on the last large-component spline when the
  orders differ (ratio Q/P = 1 at the box edge);
* the first spline and the last two splines of each component removed;
* the symmetric-definite problem solved from the lower triangle;
* states below -c^2 (the negative-energy sea) dropped; phase fixed so that the
  largest |P| coefficient is positive.

This is input generation, not part of the hot path: it runs once per ion on
the host, and its cost is never inside a timed region.
"""
from __future__ import annotations

import numpy as np
from scipy import linalg

__all__ = ["SPEED_OF_LIGHT", "dirac_matrices", "dirac_spinors", "rotated_spinors"]

#: Speed of light in atomic units, 1/alpha with alpha = 0.0072973525643 (CODATA 2018).
SPEED_OF_LIGHT = 1.0 / 0.0072973525643


def _galerkin(nv: int, b1: np.ndarray, b2: np.ndarray, weight: np.ndarray, dim: int) -> np.ndarray:
    """Matrix <B1_i | weight | B2_j> assembled from per-cell Gauss sums."""
    k1, k2 = b1.shape[2], b2.shape[2]
    cell = np.einsum("vm,vmi,vmj->vij", weight, b1, b2)
    out = np.zeros((dim, dim))
    rows = np.arange(nv)[:, None, None] + np.arange(k1)[None, :, None]
    cols = np.arange(nv)[:, None, None] + np.arange(k2)[None, None, :]
    rows = np.broadcast_to(rows, cell.shape)
    cols = np.broadcast_to(cols, cell.shape)
    keep = (rows < dim) & (cols < dim)
    np.add.at(out, (rows[keep], cols[keep]), cell[keep])
    return out


def dirac_matrices(bsp: dict, kappa: int, Z: float):
    """Hamiltonian and overlap (size 2*ns) of the point-nucleus Dirac problem."""
    c = SPEED_OF_LIGHT
    nv, gr, grw = bsp["nv"], bsp["gr"], bsp["grw"]
    ksp, ksq, nsp, nsq = bsp["ksp"], bsp["ksq"], bsp["nsp"], bsp["nsq"]
    n = max(nsp, nsq)
    bp, bq, dp, dq = bsp["bsp_p"], bsp["bsp_q"], bsp["bsp_p_d"], bsp["bsp_q_d"]

    def sym(m):
        return 0.5 * (m + m.T)

    s_pp = sym(_galerkin(nv, bp, bp, grw, n))
    s_qq = sym(_galerkin(nv, bq, bq, grw, n))
    vw = grw * (-float(Z) / gr)
    v_pp = sym(_galerkin(nv, bp, bp, vw, n))
    v_qq = sym(_galerkin(nv, bq, bq, vw, n))
    w_over_r = grw / gr
    p_dq = _galerkin(nv, bp, dq, grw, n)
    p_q_r = _galerkin(nv, bp, bq, w_over_r, n)
    if ksp != ksq:
        q_dp = _galerkin(nv, bq, dp, grw, n)
        q_p_r = _galerkin(nv, bq, bp, w_over_r, n)
    else:
        q_dp, q_p_r = p_dq, p_q_r

    H = np.zeros((2 * n, 2 * n))
    S = np.zeros((2 * n, 2 * n))
    H[:n, :n] = v_pp
    H[n:, n:] = v_qq - 2.0 * c * c * s_qq
    H[:n, n:] = -c * p_dq + kappa * c * p_q_r
    H[n:, :n] = c * q_dp + kappa * c * q_p_r
    S[:n, :n] = s_pp
    S[n:, n:] = s_qq
    if ksp != ksq:
        edge = bsp["t"][nsq]
        rn = kappa / (2.0 * edge * c)
        ip, iq = nsp - 1, n + nsq - 1
        H[ip, ip] -= rn * c
        H[ip, iq] += c
    return H, S


def dirac_spinors(bsp: dict, kappa: int, Z: float, count: int):
    """The ``count`` lowest positive-energy spinors of one kappa.

    Returns ``(P, Q, energies)`` with P, Q shaped ``(count, ns)`` (zero padded
    like atomx's ``DiracResult.get_orbital``).
    """
    c = SPEED_OF_LIGHT
    nsp, nsq = bsp["nsp"], bsp["nsq"]
    n = max(nsp, nsq)
    H, S = dirac_matrices(bsp, kappa, Z)
    keep = np.concatenate([np.arange(1, nsp - 2), np.arange(n + 1, n + nsq - 2)])
    w, v = linalg.eigh(H[np.ix_(keep, keep)], S[np.ix_(keep, keep)],
                       lower=True, driver="gvd", check_finite=False)
    physical = np.flatnonzero(w > -c * c)
    if physical.size < count:
        raise ValueError(f"basis holds only {physical.size} positive-energy states for kappa={kappa}")
    sel = physical[:count]
    full = np.zeros((2 * n, count))
    full[keep, :] = v[:, sel]
    P = np.zeros((count, n))
    Q = np.zeros((count, n))
    P[:, :nsp] = full[:nsp, :].T
    Q[:, :nsq] = full[n:n + nsq, :].T
    # Deterministic phase: the largest large-component coefficient is positive.
    idx = np.argmax(np.abs(P), axis=1)
    sign = np.where(P[np.arange(count), idx] < 0.0, -1.0, 1.0)
    return P * sign[:, None], Q * sign[:, None], w[sel]


def rotated_spinors(bsp: dict, kappa: int, Z: float, count: int, rng: np.random.Generator):
    """Seeded orthonormal rotation of the ``count`` lowest spinors of one kappa.

    The rotation is the Q factor of a QR decomposition of an N(0,1) matrix,
    with columns signed so that R has a positive diagonal.  Rotating within a
    kappa keeps the set S-orthonormal and keeps every kappa label valid.
    """
    P, Q, _ = dirac_spinors(bsp, kappa, Z, count)
    g = rng.standard_normal((count, count))
    q, r = np.linalg.qr(g)
    q = q * np.sign(np.diag(r))[None, :]
    # Spinor i of the rotated set is sum_j q[j, i] * spinor j.
    return q.T @ P, q.T @ Q
