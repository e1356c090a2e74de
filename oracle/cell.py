"""CPU oracle for the cell (bank) R^k engine — TEST INFRASTRUCTURE ONLY.

numpy-level restatement of atomx's cell algorithm (src/atomx/numerics/bspline/
convol.py) over the C loops in ``cell_oracle.c``.  Only the test-suite and the
benchmark's CPU-baseline leg use it, as the checker.

* ``get_rkb``          <- ConvolCache.get_rkb, convol.py:1507-1569 with
                          _build_rkb_sym :1684, _build_rkb_pqpq :579, _build_rkb_qpqp :593
* ``density_sym``      <- _density_sym, convol.py:713-754
* ``slater_rk_cell``   <- _compute_slater_rk_cell_once, convol.py:1788-1882
                          (the full-bank path; atomx takes it below
                          SEMISEPARABLE_DIRECT_NS = 96 splines and a factored
                          path of the same value, to ~2e-12, above it)
* ``convol_case1`` / ``convol_case4`` <- _convol_case1_t :972, _convol_case4_t :1001
* ``direct_potential_cell`` / ``exchange_matrix_cell``
                       <- compute_direct_potential_cell :1694, compute_exchange_matrix_cell :1723
* ``build_slater_rk_bilinear`` / ``slater_rk_table``
                       <- build_slater_rk_bilinear :1945 (_rkb_bilinear :1901),
                          compute_slater_rk_table :1988
* ``hf_matrix_dbsr``   <- DFSolver._build_hf_matrix_dbsr, methods/dirac_fock.py:1128-1319
                          (full-bank branches), with the density accumulations
                          of convol.py:647-710
"""
from __future__ import annotations

import ctypes

import numpy as np

from .oracle import _lib

_d = ctypes.POINTER(ctypes.c_double)
_i, _f = ctypes.c_int, ctypes.c_double

ITYPES = ("pppp", "qqqq", "pqpq", "qpqp")


def _bind():
    lib = _lib()
    if getattr(lib, "_cell_bound", False):
        return lib
    sig = {
        "oracle_gl01": [_i, _d, _d],
        "oracle_cell_moments": [_d, _d, _d, _i, _i, _i, _i, _d],
        "oracle_cell_triang": [_d, _d, _d, _d, _d, _d, _i, _i, _i, _i, _i, _i, _d],
        "oracle_cell_assemble": [_d, _d, _d, _d, _d, _i, _i, _i, _i, _d],
        "oracle_density_sym": [_d, _i, _d, _i, _i, _i, _d],
        "oracle_convol_case2": [_d, _i, _d, _i, _i, _i, _i, _d],
        "oracle_convol_case1": [_d, _d, _i, _i, _i, _d],
        "oracle_convol_case4": [_d, _d, _i, _i, _i, _i, _d],
        "oracle_rkb_bilinear": [_d, _i, _d, _d, _i, _i, _i, _i, _i, _d],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = None
    lib.oracle_sum_amb_banded.argtypes = [_d, _d, _i, _i]
    lib.oracle_sum_amb_banded.restype = _f
    lib._cell_bound = True
    return lib


def _c(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_d)


def gl01(n: int):
    x, w = np.empty(n), np.empty(n)
    _bind().oracle_gl01(n, x.ctypes.data_as(_d), w.ctypes.data_as(_d))
    return x, w


def moments(bsp, gr, grw, nv, ks, k):
    """(kk, nv) packed moments sum_m grw gr^k B_i B_j (k < 0: grw / gr^-k)."""
    bsp, pb = _c(bsp)
    gr, pg = _c(gr)
    grw, pw = _c(grw)
    out = np.empty((ks * (ks + 1) // 2, nv))
    _bind().oracle_cell_moments(pb, pg, pw, nv, gr.shape[1], ks, int(k), out.ctypes.data_as(_d))
    return out


def triang(bsp_l, bsp_r, gr, grw, t_l, t_r, nv, ks_l, ks_r, same, k):
    """(kk_l, kk_r, nv) diagonal-cell integrals (_triang_sym / _triang_pqpq)."""
    keep = [_c(a) for a in (bsp_l, bsp_r, gr, grw, t_l, t_r)]
    out = np.empty((ks_l * (ks_l + 1) // 2, ks_r * (ks_r + 1) // 2, nv))
    _bind().oracle_cell_triang(*[p for _, p in keep], nv, keep[2][0].shape[1], ks_l, ks_r, int(bool(same)), int(k),
                               out.ctypes.data_as(_d))
    return out


def _components(bd, comp):
    if comp == "p":
        return bd["bsp_p"], bd.get("tp", bd["t"]), bd.get("ksp", bd["ks"])
    return bd.get("bsp_q", bd["bsp_p"]), bd["t"], bd.get("ksq", bd["ks"])


def bank_parts(bd, k, itype):
    """Local moments and diagonal cells of one bank: (rising_l, falling_l,
    rising_r, falling_r, diag, ks_l, ks_r)."""
    left, right = itype[0], itype[1]
    bl, tl, ksl = _components(bd, left)
    br, tr, ksr = _components(bd, right)
    gr, grw, nv = bd["gr"], bd["grw"], bd["nv"]
    rl, fl = moments(bl, gr, grw, nv, ksl, k), moments(bl, gr, grw, nv, ksl, -(k + 1))
    rr, fr = (rl, fl) if left == right else (moments(br, gr, grw, nv, ksr, k), moments(br, gr, grw, nv, ksr, -(k + 1)))
    diag = triang(bl, br, gr, grw, tl, tr, nv, ksl, ksr, left == right, k)
    return rl, fl, rr, fr, diag, ksl, ksr


def get_rkb(bd, k, itype="pppp"):
    """(rkb (ns, ns, ks_l, ks_r), ns, ks_l) as ConvolCache.get_rkb returns it."""
    if itype not in ITYPES:
        raise ValueError(f"Unknown integral type: {itype}")
    rl, fl, rr, fr, diag, ksl, ksr = bank_parts(bd, k, itype)
    ns = bd["ns"]
    keep = [_c(a) for a in (rl, fl, rr, fr, diag)]
    out = np.empty((ns, ns, ksl, ksr))
    _bind().oracle_cell_assemble(*[p for _, p in keep], bd["nv"], ksl, ksr, ns, out.ctypes.data_as(_d))
    return out, ns, ksl


class Banks:
    """Bank memo per (k, itype) for one basis (the role of ConvolCache)."""

    def __init__(self, bd):
        self.bd, self._b = bd, {}

    def __call__(self, k, itype):
        key = (int(k), itype)
        if key not in self._b:
            self._b[key] = get_rkb(self.bd, k, itype)[0]
        return self._b[key]


def density_sym(p1, p2, ns, ks):
    p1, a = _c(p1)
    p2, b = _c(p2)
    out = np.empty((ns, ks))
    _bind().oracle_density_sym(a, p1.shape[0], b, p2.shape[0], ns, ks, out.ctypes.data_as(_d))
    return out


def _case2(rkb, d_left, ns_out, ks_l, ks_r):
    rkb, pr = _c(rkb)
    d_left, pd = _c(d_left)
    out = np.empty((ns_out, ks_r))
    _bind().oracle_convol_case2(pr, rkb.shape[0], pd, d_left.shape[0], ns_out, ks_l, ks_r, out.ctypes.data_as(_d))
    return out


def sum_amb_banded(a, b, ns, ks):
    a, pa = _c(a)
    b, pb = _c(b)
    assert a.shape[1] == ks and b.shape[1] == ks and a.shape[0] >= ns and b.shape[0] >= ns
    return float(_bind().oracle_sum_amb_banded(pa, pb, ns, ks))


def slater_rk_cell(Pa, Qa, Pb, Qb, Pc, Qc, Pd, Qd, bd, k, banks=None):
    """R^k(ab, cd) by the cell algorithm's full-bank path (see module doc)."""
    banks = banks or Banks(bd)
    ksp, nsp = bd.get("ksp", bd["ks"]), bd.get("nsp", bd["ns"])
    ksq, nsq = bd.get("ksq", bd["ks"]), bd.get("nsq", bd["ns"])
    ns = bd["ns"]
    r = 0.0
    r += sum_amb_banded(_case2(banks(k, "pppp"), density_sym(Pa, Pb, nsp, ksp), nsp, ksp, ksp),
                        density_sym(Pc, Pd, nsp, ksp), nsp, ksp)
    r += sum_amb_banded(_case2(banks(k, "qqqq"), density_sym(Qa, Qb, nsq, ksq), nsq, ksq, ksq),
                        density_sym(Qc, Qd, nsq, ksq), nsq, ksq)
    r += sum_amb_banded(_case2(banks(k, "pqpq"), density_sym(Pa, Pb, nsp, ksp), ns, ksp, ksq),
                        density_sym(Qc, Qd, nsq, ksq), min(ns, nsq), ksq)
    r += sum_amb_banded(_case2(banks(k, "qpqp"), density_sym(Qa, Qb, nsq, ksq), ns, ksq, ksp),
                        density_sym(Pc, Pd, nsp, ksp), min(ns, nsp), ksp)
    return r


def convol_case1(rkb, d, ns, ks_l, ks_r):
    rkb, pr = _c(rkb)
    d, pd = _c(d)
    out = np.empty((ns, ks_l))
    _bind().oracle_convol_case1(pr, pd, ns, ks_l, ks_r, out.ctypes.data_as(_d))
    return out


def convol_case4(rkb, d, ns, ks, ks_r=None, symmetric=False):
    ks_r = ks if ks_r is None else ks_r
    rkb, pr = _c(rkb)
    d, pd = _c(d)
    out = np.empty((ns, ns))
    _bind().oracle_convol_case4(pr, pd, ns, ks, ks_r, int(bool(symmetric)), out.ctypes.data_as(_d))
    return out


def banded_to_full_add(V, v, ns, ks, coeff):
    """V[i, i+s] += coeff v[i, s] and its mirror (convol.py:815-826)."""
    for s in range(ks):
        for i in range(ns - s):
            val = coeff * v[i, s]
            V[i, i + s] += val
            if s > 0:
                V[i + s, i] += val


def _orders(bd):
    return {"p": bd.get("ksp", bd["ks"]), "q": bd.get("ksq", bd["ks"])}


def density_full(p1, p2, ns):
    n1, n2 = min(p1.shape[0], ns), min(p2.shape[0], ns)
    d = np.zeros((ns, ns))
    d[:n1, :n2] = np.outer(p1[:n1], p2[:n2])
    return d


def direct_potential_cell(P, Q, bd, k, banks=None):
    banks = banks or Banks(bd)
    ns, orders = bd["ns"], _orders(bd)
    dens = {c: density_sym(v, v, ns, orders[c]) for c, v in (("p", P), ("q", Q))}
    out = []
    for a in ("p", "q"):
        banded = np.zeros((ns, orders[a]))
        for b in ("p", "q"):
            banded += convol_case1(banks(k, a + b + a + b), dens[b], ns, orders[a], orders[b])
        full = np.zeros((ns, ns))
        banded_to_full_add(full, banded, ns, orders[a], 1.0)
        out.append(full)
    return tuple(out)


def exchange_matrix_cell(aP, aQ, bP, bQ, bd, k, banks=None):
    banks = banks or Banks(bd)
    ns, orders = bd["ns"], _orders(bd)
    left, right = {"p": aP, "q": aQ}, {"p": bP, "q": bQ}
    diagonal = aP is bP and aQ is bQ
    blocks = {}
    for a, b in (("p", "p"), ("q", "q"), ("p", "q"), ("q", "p")):
        if diagonal and (a, b) == ("q", "p"):
            blocks[a, b] = blocks["p", "q"].T.copy()
            continue
        blocks[a, b] = convol_case4(banks(k, a + b + a + b), density_full(left[a], right[b], ns), ns, orders[a],
                                    orders[b], symmetric=diagonal and a == b)
    return tuple(blocks[x] for x in (("p", "p"), ("q", "q"), ("p", "q"), ("q", "p")))


def rkb_bilinear(rkb, wa, wb, n_left, n_right, ks_l, ks_r, ns_out):
    rkb, pr = _c(rkb)
    wa, pa = _c(wa)
    wb, pb = _c(wb)
    out = np.empty((ns_out, ns_out))
    _bind().oracle_rkb_bilinear(pr, rkb.shape[0], pa, pb, n_left, n_right, ks_l, ks_r, ns_out,
                                out.ctypes.data_as(_d))
    return out


def build_slater_rk_bilinear(Pa, Qa, Pb, Qb, bd, k, banks=None):
    banks = banks or Banks(bd)
    ksp, nsp = bd.get("ksp", bd["ks"]), bd.get("nsp", bd["ns"])
    ksq, nsq = bd.get("ksq", bd["ks"]), bd.get("nsq", bd["ns"])
    ns = bd["ns"]
    return (rkb_bilinear(banks(k, "pppp"), Pa, Pb, nsp, nsp, ksp, ksp, ns),
            rkb_bilinear(banks(k, "qqqq"), Qa, Qb, nsq, nsq, ksq, ksq, ns),
            rkb_bilinear(banks(k, "pqpq"), Pa, Qb, min(ns, nsp), min(ns, nsq), ksp, ksq, ns),
            rkb_bilinear(banks(k, "qpqp"), Qa, Pb, min(ns, nsq), min(ns, nsp), ksq, ksp, ns))


def slater_rk_table(M, CP_l, CQ_l, CP_r, CQ_r):
    M_PP, M_QQ, M_PQ, M_QP = M
    return CP_l.T @ M_PP @ CP_r + CQ_l.T @ M_QQ @ CQ_r + CP_l.T @ M_PQ @ CQ_r + CQ_l.T @ M_QP @ CP_r


def hf_matrix_dbsr(target, P_stack, Q_stack, ang_direct, ang_exchange, ks_list, norm, bd, banks=None,
                   skip_pq_exchange=False):
    """Fock blocks (PP, QQ, PQ, QP) of one target orbital: direct density
    sum_j a(i,j,k) d(j,j) (doubled for j = target) through case 1, exchange
    density sum_j b(i,j,k) P_i(comp) x P_j(comp) through case 4, per
    (component block, k), then symmetrised and divided by the target's norm."""
    banks = banks or Banks(bd)
    ns = bd["ns"]
    ksp, ksq = bd.get("ksp", bd["ks"]), bd.get("ksq", bd["ks"])
    hfm = {b: np.zeros((ns, ns)) for b in ("PP", "QQ", "PQ", "QP")}
    for ii, jj in ((1, 1), (1, 2), (2, 1), (2, 2)):
        block = {(1, 1): "pppp", (1, 2): "pqpq", (2, 1): "qpqp", (2, 2): "qqqq"}[ii, jj]
        ks_bra = ksp if ii == 1 else ksq
        ks_ket = ksp if jj == 1 else ksq
        comp_jj = Q_stack if jj == 2 else P_stack
        comp_ii = Q_stack if ii == 2 else P_stack
        for k in ks_list:
            a = ang_direct[target, :, k]
            b = ang_exchange[target, :, k]
            if np.any(a):
                dd = np.zeros((ns, ks_ket))
                for j in range(a.shape[0]):
                    c = a[j]
                    if c == 0.0:
                        continue
                    if j == target:
                        c = c + c
                    p = comp_jj[j]
                    dd[:, 0] += c * p * p
                    for s in range(1, ks_ket):
                        dd[:ns - s, s] += c * (p[:ns - s] * p[s:] + p[s:] * p[:ns - s])
                v = convol_case1(banks(k, block), dd, ns, ks_bra, ks_ket)
                banded_to_full_add(hfm["PP" if ii == 1 else "QQ"], v, ns, ks_bra, 1.0)
            if skip_pq_exchange and ii == 1 and jj == 2:
                continue
            if np.any(b):
                xx = np.zeros((ns, ns))
                for j in range(b.shape[0]):
                    c = b[j]
                    if c == 0.0:
                        continue
                    xx += np.outer(c * comp_ii[j], comp_jj[j])
                Kk = convol_case4(banks(k, block), xx, ns, ks_bra, ks_ket, symmetric=(ii == jj))
                hfm[{(1, 1): "PP", (1, 2): "PQ", (2, 1): "QP", (2, 2): "QQ"}[ii, jj]] += Kk
    PP = 0.5 * (hfm["PP"] + hfm["PP"].T)
    QQ = 0.5 * (hfm["QQ"] + hfm["QQ"].T)
    if skip_pq_exchange:
        PQ = hfm["QP"].T.copy()
        QP = hfm["QP"]
    else:
        PQ = 0.5 * (hfm["PQ"] + hfm["QP"].T)
        QP = PQ.T.copy()
    if norm > 1e-15:
        PP, QQ, PQ, QP = PP / norm, QQ / norm, PQ / norm, QP / norm
    return PP, QQ, PQ, QP
