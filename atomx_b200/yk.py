"""Drop-in Y^k screening functions on the dense Gauss grid (device engine).

Mirrors atomx ``numerics/yk.py``:

* ``yk_partial_matrices(n_gauss)``  (yk.py:65)  host set-up, cached per n_gauss;
* ``yk_flat(rho_flat, r_flat, w_flat, n, k, nv, ng, mo, mi)``  (yk.py:88);
* ``compute_yk(rho, gr, grw, nv, n_gauss, k)``  (yk.py:157);
* ``compute_yk_rows(rho_rows, ks, gr, grw)``  batched rows (new).

    Y^k(r) = r^{-(k+1)} int_0^r rho r'^k dr' + r^k int_r^inf rho r'^{-(k+1)} dr'

with the interpolatory partial-cell rule.  NumPy inputs return NumPy arrays
(copied to and from the device); CUDA tensors return CUDA tensors on the
current stream without host copies.  Complex c-product densities are split
into real and imaginary rows (the rule is real-linear, so the result equals
the reference's complex evaluation).  Unlike the reference, a negative or
non-integer ``k`` raises ``ValueError`` instead of silently evaluating
r^{-|k|} powers.
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np
import torch

from . import _native
from .device import as_device, is_device_tensor, resident, to_host

__all__ = ["yk_partial_matrices", "yk_flat", "compute_yk", "compute_yk_rows"]


@lru_cache(maxsize=64)
def _partial_np(n_gauss: int):
    xi, _ = np.polynomial.legendre.leggauss(n_gauss)
    leg = np.polynomial.legendre.legvander(xi, n_gauss)
    prim = np.empty((n_gauss, n_gauss))
    prim[:, 0] = xi + 1
    for ell in range(1, n_gauss):
        prim[:, ell] = (leg[:, ell + 1] - leg[:, ell - 1]) / (2 * ell + 1)
    mo = (prim * ((2 * np.arange(n_gauss) + 1) / 2)) @ leg[:, :n_gauss].T
    mi = 1 - mo
    mo.setflags(write=False)
    mi.setflags(write=False)
    return mo, mi


def yk_partial_matrices(n_gauss: int):
    """(mo, mi) with sum_j g_j mo[i, j] = int_a^{r_i} f and mi = 1 - mo.

    Built from the Legendre expansion of the cell's Lagrange basis (the same
    construction as atomx yk.py:65-84, so the matrices agree bit for bit).
    """
    n_gauss = int(n_gauss)
    if n_gauss < 1:
        raise ValueError("n_gauss must be a positive integer")
    return _partial_np(n_gauss)


def _check_k(k) -> int:
    if isinstance(k, (bool, np.bool_)) or int(k) != k or k < 0:
        raise ValueError("Slater multipole rank must be a nonnegative integer")
    return int(k)


def _device_partials(ng: int):
    mo, mi = yk_partial_matrices(ng)
    return resident(mo), resident(mi)


def _run_rows(rho2d: torch.Tensor, ks, r: torch.Tensor, w: torch.Tensor, nv: int, ng: int) -> torch.Tensor:
    """rho2d: (rows, nv*ng) float64 device tensor; ks: int or (rows,) ints."""
    L = _native.require_device()
    rows, n = rho2d.shape
    out = torch.empty_like(rho2d)
    mo, mi = _device_partials(ng)
    if isinstance(ks, (int, np.integer)) and rows == 1:
        _native.check(L.rkb_yk_flat(rho2d.data_ptr(), r.data_ptr(), w.data_ptr(), n, int(ks), nv, ng,
                                    mo.data_ptr(), mi.data_ptr(), out.data_ptr(), _native.stream_handle()),
                      "rkb_yk_flat")
        return out
    kt = torch.as_tensor(np.broadcast_to(np.asarray(ks, dtype=np.int32), (rows,)).copy(), device=rho2d.device)
    _native.check(L.rkb_yk_rows(rho2d.data_ptr(), n, kt.data_ptr(), rows, r.data_ptr(), w.data_ptr(), nv, ng,
                                mo.data_ptr(), mi.data_ptr(), out.data_ptr(), n, _native.stream_handle()),
                  "rkb_yk_rows")
    return out


def _yk_any(rho, r, w, nv: int, ng: int, ks, out_shape):
    """Dispatch real/complex and host/device inputs to the device kernel."""
    on_dev = is_device_tensor(rho)
    if on_dev:
        cplx = rho.is_complex()
    else:
        rho = np.asarray(rho)
        cplx = np.iscomplexobj(rho)
    rd = resident(r) if not is_device_tensor(r) else as_device(r)
    wd = resident(w) if not is_device_tensor(w) else as_device(w)
    n = nv * ng
    if cplx:
        if on_dev:
            rr = torch.view_as_real(rho.to(torch.complex128).reshape(-1, n).contiguous())
            parts = torch.cat([rr[..., 0], rr[..., 1]], 0).contiguous()
        else:
            arr = np.asarray(rho, dtype=np.complex128).reshape(-1, n)
            parts = as_device(np.concatenate([arr.real, arr.imag], 0))
        rows = parts.shape[0] // 2
        ks2 = ks if np.isscalar(ks) else np.concatenate([np.asarray(ks), np.asarray(ks)])
        y = _run_rows(parts, ks2, rd.reshape(-1), wd.reshape(-1), nv, ng)
        yc = torch.complex(y[:rows], y[rows:])
        return yc.reshape(out_shape) if on_dev else to_host(yc).reshape(out_shape)
    rho_d = as_device(rho).reshape(-1, n)
    y = _run_rows(rho_d, ks, rd.reshape(-1), wd.reshape(-1), nv, ng)
    return y.reshape(out_shape) if on_dev else to_host(y).reshape(out_shape)


def yk_flat(rho_flat, r_flat, w_flat, n, k, nv, ng, mo=None, mi=None):
    """Y^k of one flattened density (atomx yk.py:88 signature).

    ``mo``/``mi`` are accepted for signature compatibility; the engine uses
    its own copy of the same matrices for ``ng`` (checked when supplied).
    """
    k = _check_k(k)
    if int(n) != int(nv) * int(ng):
        raise ValueError("n must equal nv * ng")
    if mo is not None:
        ref_mo, _ = yk_partial_matrices(ng)
        if not is_device_tensor(mo) and not np.array_equal(np.asarray(mo), ref_mo):
            raise ValueError("mo does not match yk_partial_matrices(ng)")
    return _yk_any(rho_flat, r_flat, w_flat, int(nv), int(ng), k, (int(n),))


def compute_yk(rho, gr, grw, nv, n_gauss, k):
    """Y^k(r) on the (nv, n_gauss) Gauss grid (atomx yk.py:157 signature)."""
    k = _check_k(k)
    nv, n_gauss = int(nv), int(n_gauss)
    if not is_device_tensor(rho):
        rho = np.asarray(rho)
        if not np.iscomplexobj(rho):
            rho = np.asarray(rho, dtype=np.result_type(rho, np.float64))
    return _yk_any(rho, gr, grw, nv, n_gauss, k, (nv, n_gauss))


def compute_yk_rows(rho_rows, ks, gr, grw):
    """Batched Y^k: ``rho_rows`` (rows, nv*ng) with per-row multipoles ``ks``."""
    gr_shape = tuple(gr.shape)
    nv, ng = gr_shape
    ks_arr = np.asarray(ks)
    if np.any(ks_arr < 0) or not np.all(np.asarray(ks_arr, dtype=np.int64) == ks_arr):
        raise ValueError("Slater multipole ranks must be nonnegative integers")
    rows = rho_rows.shape[0]
    ks_list = int(ks_arr) if ks_arr.ndim == 0 else ks_arr.astype(np.int32)
    if np.isscalar(ks_list):
        ks_list = np.full(rows, ks_list, dtype=np.int32)
    return _yk_any(rho_rows, gr, grw, nv, ng, ks_list, (rows, nv * ng))
