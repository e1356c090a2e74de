"""Direct (Hartree) potential matrices of the Dirac-Fock driver on the device.

Drop-in for atomx ``DFSolver._build_direct_potential_yk``
(methods/dirac_fock.py:931-967), the Y^0 consumer of the path:

* the total density rho = sum occ (P^2 + Q^2) over every occupied orbital
  (``orbitals`` maps kappa to [(P coefficients, Q coefficients, occupation)],
  taken in the dict's order), minus the target orbital's own density when
  ``target_kappa``/``target_idx`` name one (dirac_fock.py:939-952);
* Y^0 = compute_yk(rho, k=0) (dirac_fock.py:954);
* V_J = <B_i | grw Y^0 | B_j> for the P basis (order ksp) and the Q basis
  (order ksq), each symmetrised as 0.5 (V + V^T) (dirac_fock.py:955-965,
  ``_assemble_integral`` numerics/bspline/integrals.py:18-56).

Orbital values come from ``rkb_eval_orbitals``, the density from
``rkb_occupied_density``, Y^0 from ``rkb_yk_rows`` and both matrices from
``rkb_bspline_sym_matrix``; nothing is computed on the host.  Returns NumPy
arrays (ns x ns) like atomx.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native
from .device import as_device, resident, to_host
from .evaluate import eval_orbitals_on_grid
from .yk import compute_yk

__all__ = ["build_direct_potential_yk", "direct_potential_yk_method"]


def _coeff_matrix(rows, ns: int) -> np.ndarray:
    out = np.zeros((max(len(rows), 1), ns))
    for i, c in enumerate(rows):
        c = np.asarray(c, dtype=np.float64).ravel()
        out[i, :min(ns, c.shape[0])] = c[:ns]
    return out


def build_direct_potential_yk(bsp_data, ns: int, orbitals, target_kappa=None, target_idx=None, ks: int | None = None):
    """(V_J_PP, V_J_QQ) of DFSolver._build_direct_potential_yk for the basis
    ``bsp_data`` (``prepare_bspline_data`` layout) and dimension ``ns``."""
    _native.require_device()
    nv = int(bsp_data["nv"])
    gr = np.asarray(bsp_data["gr"], dtype=np.float64)
    grw = np.asarray(bsp_data["grw"], dtype=np.float64)
    ng = gr.shape[1]
    ks = int(bsp_data["ks"] if ks is None else ks)
    ksp = int(bsp_data.get("ksp", ks))
    nsp = int(bsp_data.get("nsp", ns))
    ksq = int(bsp_data.get("ksq", ks))
    nsq = int(bsp_data.get("nsq", ns))
    bsp_p = bsp_data["bsp_p"]
    bsp_q = bsp_data.get("bsp_q", bsp_p)

    Ps, Qs, occ, target = [], [], [], -1
    for kappa, orb_list in orbitals.items():
        for P, Q, o in orb_list:
            Ps.append(P), Qs.append(Q), occ.append(float(o))
    if target_kappa is not None and target_idx is not None:
        lst = list(orbitals.get(target_kappa, []))
        if target_idx < len(lst):
            P, Q, _ = lst[target_idx]
            Ps.append(P), Qs.append(Q)
            target = len(Ps) - 1
            occ.append(0.0)  # counted only through the subtraction
    n = nv * ng
    L = _native.load()
    d = torch.device("cuda", torch.cuda.current_device())
    rho = torch.empty(n, dtype=torch.float64, device=d)
    if Ps:
        Pv = eval_orbitals_on_grid(as_device(_coeff_matrix(Ps, nsp)), bsp_p, nv, ksp, nsp)
        Qv = eval_orbitals_on_grid(as_device(_coeff_matrix(Qs, nsq)), bsp_q, nv, ksq, nsq)
        occ_d = as_device(np.asarray(occ))
        _native.check(L.rkb_occupied_density(Pv.data_ptr(), Qv.data_ptr(), n, len(Ps), occ_d.data_ptr(), target, n,
                                             rho.data_ptr(), _native.stream_handle()), "rkb_occupied_density")
    else:
        rho.zero_()
    y = compute_yk(rho.view(nv, ng), gr, grw, nv, ng, 0)
    w = resident(grw)
    out = []
    for bsp, kk in ((bsp_p, ksp), (bsp_q, ksq)):
        b = resident(np.ascontiguousarray(bsp, dtype=np.float64))
        V = torch.empty((int(ns), int(ns)), dtype=torch.float64, device=d)
        _native.check(L.rkb_bspline_sym_matrix(b.data_ptr(), kk, b.data_ptr(), kk, nv, ng, w.data_ptr(),
                                               y.data_ptr(), int(ns), V.data_ptr(), _native.stream_handle()),
                      "rkb_bspline_sym_matrix")
        out.append(to_host(V))
    return out[0], out[1]


def direct_potential_yk_method(self, orbitals, target_kappa=None, target_idx=None):
    """The same with atomx's method signature (reads ``self.bsp_data``,
    ``self.ns``, ``self.ks``), so ``DFSolver._build_direct_potential_yk``
    can be replaced by it."""
    return build_direct_potential_yk(self.bsp_data, self.ns, orbitals, target_kappa, target_idx, ks=self.ks)
