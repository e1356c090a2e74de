"""Arbitrary-grid trapezoid Y^k on the device: a drop-in for atomx's
numerics/quadrature.py (``yk_on_grid`` :234, ``yk_pair_dot_batch_on_grid``
:282, ``grid_slater_rk`` :394), used on fine radial grids by the scattering
and autoionization codes.

The Green action r_<^k / r_>^(k+1) is applied by two cumulative trapezoid
scans in block-scaled frames (``coulomb_tables``, after quadrature.py:190-231:
within a frame the powers are taken relative to the frame's first radius,
and carried moments change frame by a factor <= 1). The scans run on the GPU
(``rkb_grid_yk_rows`` / ``rkb_grid_pair_dot_batch``): one CTA per row, with
block-wide prefix sums inside each frame. Rows are independent. The
summation order inside a frame differs from atomx's serial loop, so values
agree with it to rounding.

Inputs may be numpy arrays (results come back as numpy, like atomx) or CUDA
tensors (results stay on the device). Errors follow atomx: a non-increasing,
non-positive or non-finite grid, or a negative or non-integer rank, raise
``ValueError``.
"""
from __future__ import annotations

import hashlib
import threading

import numpy as np
import torch

from . import _native
from .device import as_device, is_device_tensor

__all__ = ["coulomb_tables", "yk_on_grid", "yk_pair_dot_batch_on_grid", "grid_slater_rk", "GridTables"]

_lock = threading.Lock()
_cache: dict = {}


def _frame_starts(r, k_max):
    """First index of every frame, plus len(r) at the end.

    Each frame holds the points whose radius lies within a factor
    e^(128/(k_max+1)) of the frame's first radius.  Within such a frame
    (r/r0)^k and (r/r0)^-(k+1) stay inside e^(+-128) for every k <= k_max,
    far inside the double range, whatever the grid spans overall.  A frame
    always takes at least one point, so the walk ends.
    """
    log_r = np.log(r)
    width = 128.0 / (k_max + 1)
    starts = [0]
    while starts[-1] < r.shape[0]:
        first = starts[-1]
        beyond = int(np.searchsorted(log_r, log_r[first] + width, side="right"))
        starts.append(beyond if beyond > first else first + 1)
    return np.asarray(starts, dtype=np.int64)


def coulomb_tables(r, k_max):
    """(rk, inverse, cuts, transfers) of a grid, as numpy arrays.

    ``cuts`` are the frame starts (``_frame_starts``).  With r0 the first
    radius of a point's frame and x = r / r0: rk[k] = x^k and
    inverse[k] = x^-(k+1) / r0.  A moment carried from one frame to the next
    is multiplied by transfers[k][b] = (r0_b / r0_{b+1})^k, which is <= 1
    because the grid increases, so carries only shrink when they change
    frame.
    """
    if isinstance(k_max, (bool, np.bool_)) or int(k_max) != k_max or k_max < 0:
        raise ValueError('Coulomb multipole rank must be a nonnegative integer')
    k_max = int(k_max)
    r = np.asarray(r, dtype=float)
    if (r.ndim != 1 or not r.size or not np.isfinite(r).all()
            or np.any(r <= 0) or np.any(np.diff(r) <= 0)):
        raise ValueError('Coulomb grid must be finite, positive and strictly increasing')
    starts = _frame_starts(r, k_max)
    ranks = np.arange(k_max + 1)[:, None]  # integer exponents, as numpy's ** takes them
    rk = np.empty((k_max + 1, r.shape[0]))
    inverse = np.empty_like(rk)
    for lo, hi in zip(starts[:-1].tolist(), starts[1:].tolist()):
        r0 = r[lo]
        x = r[lo:hi] / r0
        # fresh results from integer exponents: numpy's vectorised pow and
        # its scalar pow can differ in the last bit, and which one runs
        # depends on the operands' types and strides
        rk[:, lo:hi] = x[None, :] ** ranks
        inverse[:, lo:hi] = x[None, :] ** (-1 - ranks) / r0
    first = r[starts[:-1]]
    transfers = (first[:-1] / first[1:])[None, :] ** ranks
    return rk, inverse, starts, transfers


class GridTables:
    """Device copies of a grid's tables for ranks 0..k_max (cached by the
    grid's content, so an edited grid never reuses stale tables)."""

    def __init__(self, r, k_max: int, device):
        r_h = np.ascontiguousarray(np.asarray(r, dtype=np.float64))
        rk, inverse, cuts, transfers = coulomb_tables(r_h, k_max)
        self.n, self.k_max, self.ncuts = r_h.shape[0], int(k_max), cuts.shape[0]
        self.ntr = max(1, transfers.shape[1])
        tr = np.zeros((k_max + 1, self.ntr))
        tr[:, :transfers.shape[1]] = transfers
        self.r = torch.as_tensor(r_h, device=device)
        self.RK = torch.as_tensor(np.ascontiguousarray(rk), device=device)
        self.inverse = torch.as_tensor(np.ascontiguousarray(inverse), device=device)
        self.cuts = torch.as_tensor(cuts, device=device)
        self.transfers = torch.as_tensor(tr, device=device)

    @staticmethod
    def get(r, k_max: int, device) -> "GridTables":
        if is_device_tensor(r):
            r = r.detach().cpu().numpy()
        r_h = np.ascontiguousarray(np.asarray(r, dtype=np.float64))
        key = (hashlib.blake2b(r_h.tobytes(), digest_size=16).hexdigest(), r_h.shape[0], str(device))
        with _lock:
            hit = _cache.get(key)
        if hit is not None and hit.k_max >= k_max:
            return hit
        tab = GridTables(r_h, max(int(k_max), hit.k_max if hit is not None else 0), device)
        with _lock:
            if len(_cache) > 64:
                _cache.clear()
            _cache[key] = tab
        return tab


def _k(k) -> int:
    if isinstance(k, (bool, np.bool_)) or int(k) != k or k < 0:
        raise ValueError('Coulomb multipole rank must be a nonnegative integer')
    return int(k)


def _i_cut(n: int, i_cut) -> int:
    return n - 1 if i_cut is None else min(int(i_cut), n - 1)


def yk_on_grid(rho, r, k, i_cut=None):
    """Y^k[rho] at grid points 0..i_cut (atomx quadrature.py:234, same arguments)."""
    k = _k(k)
    L = _native.require_device()
    on_dev = is_device_tensor(rho) or is_device_tensor(r)
    rho_d = as_device(rho).reshape(-1)
    tab = GridTables.get(r, k, rho_d.device)
    n = tab.n
    if rho_d.shape[0] != n:
        raise ValueError(f"density has {rho_d.shape[0]} points, the grid {n}")
    ic = _i_cut(n, i_cut)
    y = torch.empty(n, dtype=torch.float64, device=rho_d.device)
    ks = torch.tensor([k], dtype=torch.int64, device=rho_d.device)
    _native.check(L.rkb_grid_yk_rows(rho_d.data_ptr(), n, ks.data_ptr(), 1, tab.r.data_ptr(), n, tab.RK.data_ptr(),
                                     tab.inverse.data_ptr(), tab.cuts.data_ptr(), tab.ncuts,
                                     tab.transfers.data_ptr(), tab.ntr, ic, y.data_ptr(), n,
                                     _native.stream_handle()),
                  "rkb_grid_yk_rows")
    out = y[:ic + 1]
    return out if on_dev else out.cpu().numpy()


def yk_pair_dot_batch_on_grid(PA, QA, PB, QB, rows_a, rows_b, rows_k, rows_ok, RhoA, cons_ptr, cons_rho, r,
                              i_cut=None):
    """Batched Int rho_w(r) Y^k[rho_ab](r) dr (atomx quadrature.py:282, same
    arguments): row m forms rho = PA[a]PB[b] + QA[a]QB[b] with k = rows_k[m]
    and is dotted with RhoA[cons_rho[s]] for its consumer slots s in
    [cons_ptr[m], cons_ptr[m+1]); rows with rows_ok false leave zeros."""
    L = _native.require_device()
    on_dev = any(is_device_tensor(x) for x in (PA, QA, PB, QB, RhoA))
    cons_ptr_h = np.asarray(cons_ptr.cpu() if is_device_tensor(cons_ptr) else cons_ptr, dtype=np.int64)
    n_slots = int(cons_ptr_h[-1]) if cons_ptr_h.shape[0] else 0
    rows_k_h = np.asarray(rows_k.cpu() if is_device_tensor(rows_k) else rows_k, dtype=np.int64)
    dev = torch.device("cuda", torch.cuda.current_device())
    val = torch.zeros(n_slots, dtype=torch.float64, device=dev)
    if rows_k_h.shape[0] == 0 or n_slots == 0:
        return val if on_dev else val.cpu().numpy()
    if (rows_k_h < 0).any():
        raise ValueError('Coulomb multipole rank must be a nonnegative integer')
    tab = GridTables.get(r, int(rows_k_h.max()), dev)
    n = tab.n
    ic = _i_cut(n, i_cut)
    mats = [as_device(x) for x in (PA, QA, PB, QB)]
    ld = mats[0].shape[1] if mats[0].dim() == 2 else n
    if any(m.dim() != 2 or m.shape[1] != ld for m in mats) or ld != n:
        raise ValueError("wave rows must all have the grid's length")
    W = as_device(RhoA)
    if W.dim() != 2 or W.shape[1] < ic + 1:
        raise ValueError(f"consumer rows need at least i_cut + 1 = {ic + 1} points")
    idx = [torch.as_tensor(np.asarray(x.cpu() if is_device_tensor(x) else x, dtype=np.int64), device=dev)
           for x in (rows_a, rows_b, rows_k_h, cons_ptr_h, cons_rho)]
    ok = torch.as_tensor(np.asarray(rows_ok.cpu() if is_device_tensor(rows_ok) else rows_ok, dtype=np.uint8),
                         device=dev)
    nrows = int(rows_k_h.shape[0])
    work_rows = min(nrows, 8 * torch.cuda.get_device_properties(dev).multi_processor_count)
    work = torch.empty((work_rows, n), dtype=torch.float64, device=dev)
    _native.check(L.rkb_grid_pair_dot_batch(mats[0].data_ptr(), mats[1].data_ptr(), mats[2].data_ptr(),
                                            mats[3].data_ptr(), ld, idx[0].data_ptr(), idx[1].data_ptr(),
                                            idx[2].data_ptr(), ok.data_ptr(), nrows, W.data_ptr(), W.shape[1],
                                            idx[3].data_ptr(), idx[4].data_ptr(), tab.r.data_ptr(), n,
                                            tab.RK.data_ptr(), tab.inverse.data_ptr(), tab.cuts.data_ptr(),
                                            tab.ncuts, tab.transfers.data_ptr(), tab.ntr, ic, val.data_ptr(),
                                            work.data_ptr(), work_rows, _native.stream_handle()),
                  "rkb_grid_pair_dot_batch")
    return val if on_dev else val.cpu().numpy()


def grid_slater_rk(P_a, Q_a, P_b, Q_b, P_c, Q_c, P_d, Q_d, r_grid, k):
    """R^k(a,b,c,d) = Int rho_ac(r) Y^k[rho_bd](r) dr (atomx quadrature.py:394,
    argument order of compute_slater_rk_cell): the trapezoid rule over the
    support of rho_ac plus the half interval after its last nonzero sample
    (quadrature.py:375-391), on the device as one batched row."""
    k = _k(k)
    f = [np.asarray(x.cpu() if is_device_tensor(x) else x, dtype=np.float64) for x in
         (P_a, Q_a, P_b, Q_b, P_c, Q_c, P_d, Q_d)]
    r = np.asarray(r_grid.cpu() if is_device_tensor(r_grid) else r_grid, dtype=np.float64)
    n = r.shape[0]
    rho_ac = f[0] * f[4] + f[1] * f[5]
    nz = np.flatnonzero(rho_ac != 0.0)
    ic = min(int(nz[-1]) + 1, n - 1) if nz.size else 0
    w = np.zeros(ic + 1)
    if ic >= 1:
        dr = np.diff(r[:ic + 1])
        w[:-1] += 0.5 * dr
        w[1:] += 0.5 * dr
    W = (w * rho_ac[:ic + 1])[None, :]
    stack = np.stack
    val = yk_pair_dot_batch_on_grid(stack([f[2]]), stack([f[3]]), stack([f[6]]), stack([f[7]]), np.array([0]),
                                    np.array([0]), np.array([k]), np.array([True]), W, np.array([0, 1]),
                                    np.array([0]), r, i_cut=ic)
    return float(val[0])
