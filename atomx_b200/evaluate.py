"""Orbital values on the Gauss grid from B-spline coefficients (device engine).

Mirrors atomx ``numerics/bspline/evaluate.py``: ``eval_orbital_on_grid``
(evaluate.py:71), ``eval_P`` (:112) and ``eval_Q`` (:127) on the native grid,
kinetic-balance aware (P uses ``bsp_p`` of order ksp, Q uses ``bsp_q``).
``eval_orbitals_on_grid`` evaluates many coefficient rows in one launch.
Evaluation at caller-supplied radii (the ``radii=`` form) is a host
spline evaluation outside this path and is not provided.
"""
from __future__ import annotations

import torch

from . import _native
from .device import as_device, is_device_tensor, resident, to_host

__all__ = ["eval_orbital_on_grid", "eval_orbitals_on_grid", "eval_P", "eval_Q"]


def eval_orbitals_on_grid(coeffs, bsp, nv: int, ks: int, ns: int):
    """f[o, iv*ng + m] = sum_s c[o, iv+s] B_s(r_iv,m); returns (n_orb, nv*ng)."""
    L = _native.require_device()
    on_dev = is_device_tensor(coeffs)
    c = as_device(coeffs)
    if c.dim() == 1:
        c = c.reshape(1, -1)
    b = resident(bsp) if not is_device_tensor(bsp) else as_device(bsp)
    nv_, ng, ks_ = b.shape
    if nv_ != nv or ks_ != ks:
        raise ValueError("bsp shape does not match (nv, n_gauss, ks)")
    if c.shape[1] < ns:
        c = torch.nn.functional.pad(c, (0, ns - c.shape[1]))
    out = torch.empty((c.shape[0], nv * ng), device=c.device, dtype=torch.float64)
    _native.check(L.rkb_eval_orbitals(c.data_ptr(), c.shape[1], c.shape[0], b.data_ptr(), nv, ng, ks, ns,
                                      out.data_ptr(), nv * ng, _native.stream_handle()), "rkb_eval_orbitals")
    return out if on_dev else to_host(out)


def eval_orbital_on_grid(coeffs, bsp, nv, ks, ns):
    """Single expansion on the grid, shaped (nv, n_gauss) like atomx."""
    ng = bsp.shape[1]
    out = eval_orbitals_on_grid(coeffs, bsp, int(nv), int(ks), int(ns))
    return out.reshape(int(nv), ng)


def eval_P(coeffs, bsp_data, radii=None):
    if radii is not None:
        raise NotImplementedError("evaluation at arbitrary radii is not part of the device path")
    ksp = bsp_data.get("ksp", bsp_data["ks"])
    nsp = bsp_data.get("nsp", bsp_data["ns"])
    return eval_orbital_on_grid(coeffs, bsp_data["bsp_p"], bsp_data["nv"], ksp, nsp)


def eval_Q(coeffs, bsp_data, radii=None):
    if radii is not None:
        raise NotImplementedError("evaluation at arbitrary radii is not part of the device path")
    ksq = bsp_data.get("ksq", bsp_data["ks"])
    nsq = bsp_data.get("nsq", bsp_data["ns"])
    bsp_q = bsp_data.get("bsp_q", bsp_data["bsp_p"])
    return eval_orbital_on_grid(coeffs, bsp_q, bsp_data["nv"], ksq, nsq)
