"""Host-side radial basis set-up: knots, Gauss-Legendre cells, B-spline values.

Everything here runs once per basis on the host and produces the read-only
arrays that the device engine keeps resident (grid nodes, weights and the
B-spline values at the nodes).  The conventions follow atomx so that a
``bsp_data`` dict built here is interchangeable with atomx's own:

* knot layout of ``make_exponential_knots`` (atomx numerics/bspline/knots.py:20-45):
  ``ks`` zero knots, ``t[ks] = r_min``, geometric growth up to ``t[ns] = r_max``,
  then ``ks - 1`` more copies of ``r_max``;
* cell ``iv`` is the knot interval ``[t[ks-1+iv], t[ks+iv]]`` and carries
  ``ng`` Gauss-Legendre nodes (atomx numerics/bspline/basis.py:211-249);
* kinetic balance uses order ``ks-1`` for the large component on the same
  interior knots and order ``ks`` for the small one
  (atomx numerics/bspline/basis.py:348-438).

The B-spline values are produced by a vectorised Cox-de Boor triangle over all
nodes at once rather than a per-point loop.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "make_exponential_knots",
    "gauss_legendre_points",
    "setup_gauss_points",
    "bspline_values",
    "knots_for_order",
    "prepare_bspline_data",
]


def make_exponential_knots(ns: int, ks: int, r_min: float, r_max: float) -> np.ndarray:
    """Geometric knot sequence of length ``ns + ks``.

    Interior breakpoints grow by the constant ratio ``(r_max/r_min)^(1/(nv-1))``
    with ``nv = ns - ks + 1`` cells; the first cell is ``[0, r_min]``.  The
    breakpoints are accumulated by repeated multiplication, the same recurrence
    atomx uses (knots.py:39-41), so both sequences agree bit for bit.
    """
    nv = ns - ks + 1
    if nv < 2 or ks < 1 or not (0.0 < r_min < r_max):
        raise ValueError("need ns - ks + 1 >= 2, ks >= 1 and 0 < r_min < r_max")
    ratio = np.exp(np.log(r_max / r_min) / (nv - 1))
    t = np.zeros(ns + ks)
    value = float(r_min)
    t[ks] = value
    for i in range(ks + 1, ns + 1):
        value = value * ratio
        t[i] = value
    t[ns:] = r_max
    return t


def gauss_legendre_points(n: int):
    """Nodes and weights of the ``n``-point Gauss-Legendre rule on [-1, 1]."""
    return np.polynomial.legendre.leggauss(int(n))


def setup_gauss_points(t: np.ndarray, ns: int, ks: int, n_gauss: int | None = None):
    """Per-cell nodes ``gr`` and weights ``grw``, both shaped ``(nv, n_gauss)``."""
    if n_gauss is None:
        n_gauss = ks
    nv = ns - ks + 1
    xi, wi = gauss_legendre_points(n_gauss)
    left = np.asarray(t[ks - 1:ks - 1 + nv], dtype=np.float64)
    right = np.asarray(t[ks:ks + nv], dtype=np.float64)
    half = 0.5 * (right - left)
    mid = 0.5 * (left + right)
    gr = mid[:, None] + half[:, None] * xi[None, :]
    grw = half[:, None] * wi[None, :]
    return gr, grw


def _cox_de_boor(t: np.ndarray, order: int, x: np.ndarray, left: np.ndarray) -> np.ndarray:
    """Values of the ``order`` non-zero B-splines at each point.

    ``left[p]`` is the knot index with ``t[left] <= x[p] < t[left+1]``.  Row
    ``p`` of the result holds B_{left-order+1..left}(x[p]).
    """
    npts = x.shape[0]
    b = np.zeros((npts, order))
    b[:, 0] = 1.0
    right_gap = np.zeros((npts, order))
    left_gap = np.zeros((npts, order))
    for j in range(1, order):
        right_gap[:, j] = t[left + j] - x
        left_gap[:, j] = x - t[left + 1 - j]
        carry = np.zeros(npts)
        for r in range(j):
            frac = b[:, r] / (right_gap[:, r + 1] + left_gap[:, j - r])
            b[:, r] = carry + right_gap[:, r + 1] * frac
            carry = left_gap[:, j - r] * frac
        b[:, j] = carry
    return b


def bspline_values(t: np.ndarray, ns: int, ks: int, gr: np.ndarray, with_derivative: bool = True):
    """B-spline values (and first derivatives) at every cell node.

    Returns ``(val, der)`` with shapes ``(nv, ng, ks)``; ``val[iv, m, s]`` is
    B_{iv+s}(gr[iv, m]).  The derivative uses the order-lowering identity
    B'_{i,k} = (k-1) [B_{i,k-1}/(t_{i+k-1}-t_i) - B_{i+1,k-1}/(t_{i+k}-t_{i+1})].
    """
    nv, ng = gr.shape
    x = gr.reshape(-1)
    left = np.repeat(np.arange(ks - 1, ks - 1 + nv), ng)
    val = _cox_de_boor(t, ks, x, left).reshape(nv, ng, ks)
    if not with_derivative:
        return val, None
    km = ks - 1
    der = np.zeros((nv * ng, ks))
    if km >= 1:
        low = _cox_de_boor(t, km, x, left)  # B_{left-km+1..left} of order km
        for i in range(ks):
            g = left - ks + 1 + i  # global index of B_i (order ks)
            lo = np.zeros(nv * ng)
            hi = np.zeros(nv * ng)
            if 1 <= i <= km:
                den = t[g + km] - t[g]
                ok = np.abs(den) > 1e-30
                lo[ok] = low[ok, i - 1] / den[ok]
            if i < km:
                den = t[g + ks] - t[g + 1]
                ok = np.abs(den) > 1e-30
                hi[ok] = low[ok, i] / den[ok]
            der[:, i] = km * (lo - hi)
    return val, der.reshape(nv, ng, ks)


def knots_for_order(t: np.ndarray, ks: int, ns: int, order: int):
    """Knot sequence of another order on the same interior breakpoints."""
    nv = ns - ks + 1
    n_target = nv + order - 1
    interior = t[ks:ns]
    out = np.empty(n_target + order)
    out[:order] = t[0]
    out[order:order + interior.shape[0]] = interior
    out[n_target:] = t[ns]
    return out, n_target


def prepare_bspline_data(t: np.ndarray, ns: int, ks: int, n_gauss: int | None = None,
                         kinetic_balance: bool = False) -> dict:
    """Build an atomx-compatible ``bsp_data`` dict for one radial basis.

    Keys: nv, ks, ksp, ksq, nsp, nsq, ns, gr, grw, bsp_p, bsp_q, bsp_p_d,
    bsp_q_d, t, tp — the same names and shapes as atomx's
    ``prepare_bspline_data`` (basis.py:364-438).
    """
    t = np.asarray(t, dtype=np.float64)
    nv = ns - ks + 1
    gr, grw = setup_gauss_points(t, ns, ks, n_gauss)
    ksq = ks
    ksp = ks - 1 if kinetic_balance else ks
    nsq = nv + ksq - 1
    nsp = nv + ksp - 1
    bsp_q, bsp_q_d = bspline_values(t, nsq, ksq, gr)
    if ksp == ksq:
        tp = t
        bsp_p, bsp_p_d = bsp_q.copy(), bsp_q_d.copy()
    else:
        tp, n_check = knots_for_order(t, ks, ns, ksp)
        assert n_check == nsp
        bsp_p, bsp_p_d = bspline_values(tp, nsp, ksp, gr)
    return {
        "nv": nv, "ks": ks, "ksp": ksp, "ksq": ksq, "nsp": nsp, "nsq": nsq,
        "gr": gr, "grw": grw, "bsp_p": bsp_p, "bsp_q": bsp_q,
        "bsp_p_d": bsp_p_d, "bsp_q_d": bsp_q_d, "t": t, "tp": tp,
        "ns": max(nsp, nsq),
    }
