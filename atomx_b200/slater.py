"""Drop-in Slater integrals R^k from pre-built densities (device engine).

Mirrors atomx ``numerics/bspline/slater.py``:

* ``slater_rk_poisson(rho13, rho24, gr, grw, nv, n_gauss, k)``  (slater.py:118)
  R^k = sum_i w_i rho13_i Y^k[rho24]_i, O(N) per integral;
* ``slater_rk_direct(rho13, rho24, gr, grw, k)``  (slater.py:81) the O(N^2)
  double quadrature with every coincident cell split along r = s;
* ``slater_rk(rho13, rho24, bsp_data, k, method="poisson")``  (slater.py:133);
* ``slater_rk_poisson_batch(rho13_rows, rho24_rows, gr, grw, k)`` (new): one
  launch for many integrals.

    R^k(13, 24) = int int rho13(r1) r_<^k / r_>^{k+1} rho24(r2) dr1 dr2

Errors follow the reference: ``ValueError`` for an unknown method, a grid
that is not 2-D, or a negative / non-integer rank.
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np
import torch

from . import _native
from .device import as_device, is_device_tensor, resident
from .yk import _check_k, compute_yk

__all__ = ["DEFAULT_METHOD", "AVAILABLE_METHODS", "slater_rk_poisson", "slater_rk_direct", "slater_rk",
           "slater_rk_poisson_batch"]

#: Integrator used when the caller does not specify one.
DEFAULT_METHOD = "poisson"
#: Names accepted by :func:`slater_rk`.
AVAILABLE_METHODS = ("poisson", "direct")


def _dots(a: torch.Tensor, b: torch.Tensor, w: torch.Tensor) -> torch.Tensor:
    """out[e] = sum_i w_i a[e, i] b[e, i] for real row-aligned a, b (device)."""
    L = _native.require_device()
    rows, n = a.shape
    idx = torch.arange(rows, device=a.device, dtype=torch.int64)
    out = torch.empty(rows, device=a.device, dtype=torch.float64)
    _native.check(L.rkb_weighted_dots(a.data_ptr(), n, b.data_ptr(), n, w.data_ptr(), n, idx.data_ptr(),
                                      idx.data_ptr(), rows, out.data_ptr(), _native.stream_handle()),
                  "rkb_weighted_dots")
    return out


def _as_rows(x, n):
    if is_device_tensor(x):
        return x.reshape(-1, n)
    return np.asarray(x).reshape(-1, n)


def _contract(rho13, y, grw):
    """sum(grw * rho13 * y) per row, complex-aware; returns a device tensor."""
    wd = resident(grw).reshape(-1) if not is_device_tensor(grw) else as_device(grw).reshape(-1)
    n = wd.shape[0]
    cplx = (rho13.is_complex() if is_device_tensor(rho13) else np.iscomplexobj(rho13)) or \
        (y.is_complex() if is_device_tensor(y) else np.iscomplexobj(y))
    if not cplx:
        return _dots(as_device(_as_rows(rho13, n)), as_device(_as_rows(y, n)), wd)
    a = as_device(_as_rows(rho13, n), dtype=torch.complex128)
    b = as_device(_as_rows(y, n), dtype=torch.complex128)
    ar, ai, br, bi = a.real.contiguous(), a.imag.contiguous(), b.real.contiguous(), b.imag.contiguous()
    re = _dots(ar, br, wd) - _dots(ai, bi, wd)
    im = _dots(ar, bi, wd) + _dots(ai, br, wd)
    return torch.complex(re, im)


def _scalar(t: torch.Tensor):
    v = t.reshape(-1)[0].item()
    return v


def slater_rk_poisson(rho13, rho24, gr, grw, nv, n_gauss, k):
    """Fast O(N) Slater integral via the Y^k screening function of ``rho24``."""
    k = _check_k(k)
    nv, n_gauss = int(nv), int(n_gauss)
    y = compute_yk(rho24.reshape(nv, n_gauss) if hasattr(rho24, "reshape") else np.reshape(rho24, (nv, n_gauss)),
                   gr, grw, nv, n_gauss, k)
    return _scalar(_contract(rho13, y, grw))


def slater_rk_poisson_batch(rho13_rows, rho24_rows, gr, grw, k):
    """R^k for many (rho13, rho24) row pairs in one launch; returns (rows,)."""
    k = _check_k(k)
    nv, ng = tuple(gr.shape)
    from .yk import compute_yk_rows
    y = compute_yk_rows(rho24_rows, k, gr, grw)
    out = _contract(rho13_rows, y, grw)
    return out if is_device_tensor(rho13_rows) else out.cpu().numpy()


@lru_cache(maxsize=16)
def _triangle_rule(n_gauss: int, order: int):
    """Gauss nodes of the split coincident cell and the density interpolants.

    On a cell's lower triangle r = a + h x, s = a + h x y (x, y in (0,1)); the
    Jacobian h^2 x cancels the Coulomb corner.  ``outer`` interpolates the node
    values at r, ``inner`` at s (Legendre interpolation of degree ng-1), as in
    atomx slater.py:63-78.
    """
    nodes, _ = np.polynomial.legendre.leggauss(n_gauss)
    x, w = np.polynomial.legendre.leggauss(order)
    x, w = (x + 1) / 2, w / 2
    inverse = np.linalg.solve(np.polynomial.legendre.legvander(nodes, n_gauss - 1), np.eye(n_gauss))
    outer = np.polynomial.legendre.legvander(2 * x - 1, n_gauss - 1) @ inverse
    inner = np.polynomial.legendre.legvander(2 * x[:, None] * x[None, :] - 1, n_gauss - 1) @ inverse
    return nodes, x, w, np.ascontiguousarray(outer), np.ascontiguousarray(inner.reshape(order * order, n_gauss))


def slater_rk_direct(rho13, rho24, gr, grw, k):
    """Independent O(N^2) double quadrature, split along each cell's r = s cusp."""
    gr_np = gr if is_device_tensor(gr) else np.asarray(gr)
    grw_np = grw if is_device_tensor(grw) else np.asarray(grw)
    if gr_np.ndim != 2 or tuple(gr_np.shape) != tuple(grw_np.shape):
        raise ValueError("direct Slater integration requires a 2-D cell Gauss grid and weights")
    if isinstance(k, (bool, np.bool_)) or k < 0 or int(k) != k:
        raise ValueError("Slater multipole rank must be a nonnegative integer")
    k = int(k)
    nv, ng = tuple(gr_np.shape)
    order = max(2 * ng, (k + ng + 1) // 2)
    nodes, x, wx, outer, inner = _triangle_rule(ng, order)
    L = _native.require_device()
    cplx = any((t.is_complex() if is_device_tensor(t) else np.iscomplexobj(t)) for t in (rho13, rho24))
    rd, wd = resident(gr_np) if not is_device_tensor(gr_np) else as_device(gr_np), \
        resident(grw_np) if not is_device_tensor(grw_np) else as_device(grw_np)
    xd, wxd, od, idd = resident(x), resident(wx), resident(outer), resident(inner)

    def run(a, b):
        out = torch.empty(1, device=rd.device, dtype=torch.float64)
        _native.check(L.rkb_slater_direct(a.data_ptr(), b.data_ptr(), rd.data_ptr(), wd.data_ptr(), nv, ng, k,
                                          order, float(nodes[0]), xd.data_ptr(), wxd.data_ptr(), od.data_ptr(),
                                          idd.data_ptr(), out.data_ptr(), _native.stream_handle()),
                      "rkb_slater_direct")
        return out

    if not cplx:
        return _scalar(run(as_device(rho13).reshape(-1), as_device(rho24).reshape(-1)))
    a = as_device(rho13, dtype=torch.complex128).reshape(-1)
    b = as_device(rho24, dtype=torch.complex128).reshape(-1)
    ar, ai, br, bi = (t.contiguous() for t in (a.real, a.imag, b.real, b.imag))
    re = run(ar, br) - run(ai, bi)
    im = run(ar, bi) + run(ai, br)
    return complex(_scalar(re), _scalar(im))


def slater_rk(rho13, rho24, bsp_data: dict, k: int, method: str = DEFAULT_METHOD):
    """Slater radial integral R^k(13, 24) with a selectable integrator."""
    gr = bsp_data["gr"]
    grw = bsp_data["grw"]
    nv = bsp_data["nv"]
    n_gauss = gr.shape[1]
    if method == "poisson":
        return slater_rk_poisson(rho13, rho24, gr, grw, nv, n_gauss, k)
    if method == "direct":
        return slater_rk_direct(rho13, rho24, gr, grw, k)
    raise ValueError(f"unknown Slater integrator {method!r}; choose from {AVAILABLE_METHODS}")
