"""Coefficient-level Slater integrals R^k, F^k, G^k (device engine).

Mirrors atomx ``numerics/bspline/slater_yk.py``:

* ``compute_slater_rk(Pa, Qa, Pb, Qb, Pc, Qc, Pd, Qd, bsp_data, k)`` (:159)
  R^k(ab, cd) = int rho_ab Y^k[rho_cd] dr with rho_ab = P_a P_b + Q_a Q_b —
  note the argument convention: densities are formed from positions (1,2)
  and (3,4), not (1,3) and (2,4);
* ``compute_slater_fk`` (:199) F^k(a,b) = R^k(aa, bb);
* ``compute_slater_gk`` (:205) G^k(a,b) = R^k(ab, ba).

The eight orbital evaluations run as two batched launches (P and Q
components), followed by the pair densities, one Y^k row and one dot.

* ``compute_exchange_matrix(orb_b_P, orb_b_Q, bsp_data, k)`` (:125) the
  non-local exchange matrices K^k_PP (nsp x nsp, order-ksp basis) and K^k_QQ
  (nsq x nsq, order-ksq basis) of ``_exchange_matrix_kernel`` (:34-122),
  whose Y^k uses rectangle-rule cumulative sums: one ``rkb_exchange_matrix``
  launch per block, one block per matrix column.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native
from .device import as_device, resident
from .evaluate import eval_orbitals_on_grid
from .slater import _dots
from .yk import _check_k, _run_rows

__all__ = ["compute_slater_rk", "compute_slater_fk", "compute_slater_gk", "compute_exchange_matrix"]


def compute_slater_rk(Pa, Qa, Pb, Qb, Pc, Qc, Pd, Qd, bsp_data, k):
    k = _check_k(k)
    _native.require_device()
    nv = bsp_data["nv"]
    gr, grw = bsp_data["gr"], bsp_data["grw"]
    ng = gr.shape[1]
    ksp = bsp_data.get("ksp", bsp_data["ks"])
    nsp = bsp_data.get("nsp", bsp_data["ns"])
    ksq = bsp_data.get("ksq", bsp_data["ks"])
    nsq = bsp_data.get("nsq", bsp_data["ns"])
    bsp_q = bsp_data.get("bsp_q", bsp_data["bsp_p"])
    width_p = max(len(v) for v in (Pa, Pb, Pc, Pd))
    width_q = max(len(v) for v in (Qa, Qb, Qc, Qd))
    cp = np.zeros((4, max(width_p, nsp)))
    cq = np.zeros((4, max(width_q, nsq)))
    for i, v in enumerate((Pa, Pb, Pc, Pd)):
        cp[i, :len(v)] = v
    for i, v in enumerate((Qa, Qb, Qc, Qd)):
        cq[i, :len(v)] = v
    f = eval_orbitals_on_grid(as_device(cp), resident(bsp_data["bsp_p"]), nv, ksp, nsp)
    g = eval_orbitals_on_grid(as_device(cq), resident(bsp_q), nv, ksq, nsq)
    rho_ab = f[0] * f[1] + g[0] * g[1]
    rho_cd = (f[2] * f[3] + g[2] * g[3]).reshape(1, -1).contiguous()
    r = resident(gr).reshape(-1)
    w = resident(grw).reshape(-1)
    y = _run_rows(rho_cd, k, r, w, nv, ng)
    return float(_dots(rho_ab.reshape(1, -1).contiguous(), y, w)[0].item())


def compute_slater_fk(orb_a_P, orb_a_Q, orb_b_P, orb_b_Q, bsp_data, k):
    """Direct Slater integral F^k(a, b) = R^k(aa, bb)."""
    return compute_slater_rk(orb_a_P, orb_a_Q, orb_a_P, orb_a_Q, orb_b_P, orb_b_Q, orb_b_P, orb_b_Q, bsp_data, k)


def compute_slater_gk(orb_a_P, orb_a_Q, orb_b_P, orb_b_Q, bsp_data, k):
    """Exchange Slater integral G^k(a, b) = R^k(ab, ba)."""
    return compute_slater_rk(orb_a_P, orb_a_Q, orb_b_P, orb_b_Q, orb_b_P, orb_b_Q, orb_a_P, orb_a_Q, bsp_data, k)


def compute_exchange_matrix(orb_b_P, orb_b_Q, bsp_data, k):
    """(K_PP, K_QQ) as atomx compute_exchange_matrix (slater_yk.py:125-155)."""
    if isinstance(k, bool) or int(k) != k or k < 0:
        raise ValueError(f"k must be a non-negative integer (got {k!r})")
    k = int(k)
    L = _native.require_device()
    nv = int(bsp_data["nv"])
    ns = int(bsp_data["ns"])
    gr, grw = bsp_data["gr"], bsp_data["grw"]
    ng = gr.shape[1]
    r, w = resident(np.asarray(gr).ravel()), resident(np.asarray(grw).ravel())
    bsp_p = bsp_data["bsp_p"]
    blocks = ((orb_b_P, bsp_p, int(bsp_data.get("ksp", bsp_data["ks"])), int(bsp_data.get("nsp", ns))),
              (orb_b_Q, bsp_data.get("bsp_q", bsp_p), int(bsp_data.get("ksq", bsp_data["ks"])),
               int(bsp_data.get("nsq", ns))))
    out = []
    for coeffs, bsp, ks, nsb in blocks:
        fb = eval_orbitals_on_grid(as_device(np.asarray(coeffs, dtype=np.float64)), bsp, nv, ks, nsb)
        b = resident(np.ascontiguousarray(bsp, dtype=np.float64))
        K = torch.empty((nsb, nsb), dtype=torch.float64, device=fb.device)
        _native.check(L.rkb_exchange_matrix(fb.data_ptr(), b.data_ptr(), r.data_ptr(), w.data_ptr(), nv, ng, ks, nsb,
                                            k, K.data_ptr(), _native.stream_handle()), "rkb_exchange_matrix")
        out.append(K.cpu().numpy())
    return out[0], out[1]
