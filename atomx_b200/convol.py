"""Cell (bank) R^k engine on the device: a drop-in for atomx's
numerics/bspline/convol.py (the DBSR_HF cell algorithm used by the CI, MBPT
and Dirac-Fock Fock-matrix paths).

The banks rkb[i][j][ip][jp] (four-index integrals of B-spline products,
ConvolCache.get_rkb, convol.py:1507) are built on the device by
``rkb_cell_moments`` / ``rkb_cell_diag`` / ``rkb_cell_assemble`` and stay
there, one block matrix per multipole:

    K_full = [[K_pp, K_pq], [K_qp, K_qq]],  K_xy[(ip, i)][(jp, j)] = rkb_xyxy[i][j][ip][jp]

(each component block padded to a multiple of 16 columns).  With the banded
pair densities of _density_sym in the same index order,
D(ab) = [D_P(ab) | D_Q(ab)], the cell integral of atomx's
compute_slater_rk_cell (convol.py:1756) is the bilinear form

    R^k(ab, cd) = D(ab) K_full D(cd)^T,

so a batch of integrals is one FP64 GEMM W = D_right K_full^T over the
distinct right pairs plus one gathered dot per integral, and a whole table is
that GEMM plus a symmetric table contraction.  The same W rows are the pair
potentials of the CI radial evaluator (physics/csf/matrix.py:703) and, with
the exchange contraction (_convol_case4_t) and the density accumulations,
give the DBSR Fock blocks of DFSolver._build_hf_matrix_dbsr
(methods/dirac_fock.py:1128).

The banks equal atomx's bit for bit (same operations in the same order); the
contractions sum in another order and agree to rounding.  atomx switches its
scalar integrals to a factored ("semiseparable") CPU path above
SEMISEPARABLE_DIRECT_NS splines; that path equals the full bank to ~2e-12,
and the device uses the full bank at every size.

Inputs are numpy arrays (results come back as numpy, as from atomx) or CUDA
tensors where noted.  Errors follow atomx: an unknown integral type raises
``ValueError``, a non-finite cell integral ``FloatingPointError``.
"""
from __future__ import annotations

import threading
from collections import OrderedDict
from collections.abc import Mapping
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native
from .device import as_device, resident, to_host

__all__ = ["ConvolCache", "CellBank", "grid_bank_key", "shared_banks", "SEMISEPARABLE_DIRECT_NS",
           "compute_slater_rk_cell", "compute_slater_fk_cell", "compute_slater_gk_cell",
           "compute_slater_rk_cell_batch", "build_slater_rk_bilinear", "eval_slater_rk_bilinear",
           "compute_slater_rk_table", "compute_direct_potential_cell", "compute_exchange_matrix_cell",
           "cell_densities", "cell_tables", "build_hf_matrix_dbsr", "build_hf_matrices_dbsr",
           "bspline_pair_potential", "PairPotentials", "radial_evaluator"]

#: atomx's switch to its factored scalar path (kept for API parity; the device
#: engine evaluates the full bank at every size)
SEMISEPARABLE_DIRECT_NS = 96
ITYPES = ("pppp", "qqqq", "pqpq", "qpqp")
_BANK_CACHE_LIMIT = 4
_banks: OrderedDict = OrderedDict()
_banks_lock = threading.Lock()


def _round16(x: int) -> int:
    return (x + 15) // 16 * 16


def grid_bank_key(bsp_data):
    """Content key of the banks built on ``bsp_data``: the knot sequences,
    orders and sizes and the quadrature shape (atomx convol.py:1415)."""
    if not isinstance(bsp_data, Mapping) or bsp_data.get("t") is None:
        raise TypeError("ConvolCache needs a B-spline workspace mapping carrying a 't' knot vector "
                        f"(got {type(bsp_data).__name__})")
    t = np.ascontiguousarray(bsp_data["t"], dtype=np.float64)
    tp = bsp_data.get("tp")
    tp_b = b"" if tp is None or np.array_equal(tp, t) else np.ascontiguousarray(tp, dtype=np.float64).tobytes()
    ks = int(bsp_data.get("ks", bsp_data.get("ksq", 0)))
    gr = bsp_data.get("gr")
    return (int(bsp_data["nv"]), ks, int(bsp_data.get("ksp", ks)), int(bsp_data.get("ksq", ks)),
            int(bsp_data.get("nsp", bsp_data.get("ns", 0))), int(bsp_data.get("nsq", bsp_data.get("ns", 0))),
            int(bsp_data.get("ns", 0)), t.shape, t.tobytes(), tp_b, None if gr is None else tuple(np.shape(gr)))


def shared_banks(bsp_data, key=None) -> dict:
    """The process-wide bank dict of one grid (LRU over a few grids)."""
    key = grid_bank_key(bsp_data) if key is None else key
    with _banks_lock:
        d = _banks.get(key)
        if d is None:
            d = _banks[key] = {}
            while len(_banks) > _BANK_CACHE_LIMIT:
                _banks.popitem(last=False)
        else:
            _banks.move_to_end(key)
        return d


@dataclass
class CellBank:
    """Device banks of one multipole: K_full and the pieces it came from."""
    k: int
    ns: int
    ksp: int
    ksq: int
    kp_pad: int               # columns of the P block (multiple of 16)
    kq_pad: int
    K: torch.Tensor           # (kdim, kdim) block matrix, kdim = kp_pad + kq_pad
    moments: dict = field(default_factory=dict)   # ("p"|"q", "rising"|"falling") -> (kk, nv)

    @property
    def kdim(self) -> int:
        return self.kp_pad + self.kq_pad

    def offsets(self, itype: str):
        """(row offset, column offset, ks_left, ks_right) of one bank block."""
        if itype not in ITYPES:
            raise ValueError(f"Unknown integral type: {itype}")
        left, right = itype[0], itype[1]
        return ((0 if left == "p" else self.kp_pad), (0 if right == "p" else self.kp_pad),
                self.ksp if left == "p" else self.ksq, self.ksp if right == "p" else self.ksq)

    def block(self, itype: str) -> torch.Tensor:
        """(ks_l * ns, ks_r * ns) view of one bank in K layout."""
        r0, c0, ksl, ksr = self.offsets(itype)
        return self.K[r0:r0 + ksl * self.ns, c0:c0 + ksr * self.ns]


def _gl01(n: int):
    L = _native.load()
    x, w = np.empty(n), np.empty(n)
    L.rkb_gauss_legendre_01(n, x.ctypes.data, w.ctypes.data)
    return x, w


def _orders(bd):
    return {"p": int(bd.get("ksp", bd["ks"])), "q": int(bd.get("ksq", bd["ks"]))}


class ConvolCache:
    """Device banks of one basis, shared by every cache on equal-content grids
    (atomx convol.py:1478).  ``bank(k)`` is the device block matrix;
    ``get_rkb`` / ``get_rkb_t`` return host copies in atomx's layouts."""

    def __init__(self, bsp_data):
        self.bsp_data = bsp_data
        self.grid_key = grid_bank_key(bsp_data)
        self._cache = shared_banks(bsp_data, self.grid_key)
        self._lock = threading.Lock()

    def same_grid(self, bsp_data) -> bool:
        try:
            return grid_bank_key(bsp_data) == self.grid_key
        except (KeyError, TypeError):
            return False

    # ------------------------------------------------------------ building
    def bank(self, k: int, stream=None) -> CellBank:
        k = int(k)
        if k < 0:
            raise ValueError("multipole rank must be a nonnegative integer")
        dkey = (k, torch.cuda.current_device())
        with self._lock:
            hit = self._cache.get(dkey)
            if hit is None:
                hit = self._cache[dkey] = self._build(k, stream)
        return hit

    def _build(self, k: int, stream=None) -> CellBank:
        L = _native.require_device()
        bd = self.bsp_data
        s = _native.stream_handle(stream)
        nv, ns = int(bd["nv"]), int(bd["ns"])
        gr, grw = resident(bd["gr"]), resident(bd["grw"])
        ng = int(gr.shape[1])
        o = _orders(bd)
        comp = {"p": (resident(bd["bsp_p"]), resident(bd.get("tp", bd["t"]))),
                "q": (resident(bd.get("bsp_q", bd["bsp_p"])), resident(bd["t"]))}
        dev = gr.device
        kp_pad, kq_pad = _round16(o["p"] * ns), _round16(o["q"] * ns)
        K = torch.zeros((kp_pad + kq_pad, kp_pad + kq_pad), dtype=torch.float64, device=dev)
        bank = CellBank(k=k, ns=ns, ksp=o["p"], ksq=o["q"], kp_pad=kp_pad, kq_pad=kq_pad, K=K)
        for c in ("p", "q"):
            b, _ = comp[c]
            kk = o[c] * (o[c] + 1) // 2
            for name, power in (("rising", k), ("falling", -(k + 1))):
                m = torch.empty((kk, nv), dtype=torch.float64, device=dev)
                _native.check(L.rkb_cell_moments(b.data_ptr(), gr.data_ptr(), grw.data_ptr(), nv, ng, o[c], power,
                                                 m.data_ptr(), s), "rkb_cell_moments")
                bank.moments[c, name] = m
        for itype in ITYPES:
            left, right = itype[0], itype[1]
            (bl, tl), (br, tr) = comp[left], comp[right]
            ksl, ksr = o[left], o[right]
            same = left == right
            n_sub = (ksl if same else max(ksl, ksr)) + k // 2
            x, w = _gl01(n_sub)
            x01, w01 = resident(x), resident(w)
            diag = torch.empty((ksl * (ksl + 1) // 2, ksr * (ksr + 1) // 2, nv), dtype=torch.float64, device=dev)
            _native.check(L.rkb_cell_diag(bl.data_ptr(), br.data_ptr(), gr.data_ptr(), grw.data_ptr(), tl.data_ptr(),
                                          tr.data_ptr(), nv, ng, ksl, ksr, int(same), k, x01.data_ptr(),
                                          w01.data_ptr(), n_sub, diag.data_ptr(), s), "rkb_cell_diag")
            r0, c0, _, _ = bank.offsets(itype)
            m = bank.moments
            _native.check(L.rkb_cell_assemble(m[left, "rising"].data_ptr(), m[left, "falling"].data_ptr(),
                                              m[right, "rising"].data_ptr(), m[right, "falling"].data_ptr(),
                                              diag.data_ptr(), nv, ksl, ksr, ns, K.data_ptr(), K.shape[1], r0, c0, s),
                          "rkb_cell_assemble")
        return bank

    # ------------------------------------------------------- atomx layouts
    def get_rkb(self, k, itype="pppp"):
        """(rkb (ns, ns, ks_l, ks_r) host array, ns, ks_l) as atomx returns it."""
        b = self.bank(k)
        _, _, ksl, ksr = b.offsets(itype)
        blk = to_host(b.block(itype).contiguous()).reshape(ksl, b.ns, ksr, b.ns)
        return np.ascontiguousarray(blk.transpose(1, 3, 0, 2)), b.ns, ksl

    def get_rkb_t(self, k, itype="pppp"):
        """(rkbT (ks_l, ks_r, ns, ns) host array, ns, ks_l): rkbT[ip, jp, i, j] = rkb[i, j, ip, jp]."""
        b = self.bank(k)
        _, _, ksl, ksr = b.offsets(itype)
        blk = to_host(b.block(itype).contiguous()).reshape(ksl, b.ns, ksr, b.ns)
        return np.ascontiguousarray(blk.transpose(0, 2, 1, 3)), b.ns, ksl

    def _pair_moments(self, k, comp):
        """Global pair moments (ks, ns) of one component: the cell moments of
        each upper B-spline pair summed over its cells in ascending order."""
        b = self.bank(k)
        ks = b.ksp if comp == "p" else b.ksq
        out = []
        for name in ("rising", "falling"):
            local = to_host(b.moments[comp, name])
            nv = local.shape[1]
            glob = np.zeros((ks, b.ns))
            for iv in range(nv):
                pair = 0
                for first in range(ks):
                    for second in range(first, ks):
                        i = iv + first
                        if i + second - first < b.ns:
                            glob[second - first, i] += local[pair, iv]
                        pair += 1
            out.append(glob)
        return out

    def get_coulomb_factors(self, k, itype="pppp"):
        """(near, rising_left, falling_left, rising_right, falling_right) as
        atomx's ConvolCache.get_coulomb_factors (convol.py:1613): the bank
        entries of overlapping pair supports, near[ip, jp, i, j - (i + ip -
        ks_l + 1)], and the global pair moments of both components."""
        if itype not in ITYPES:
            raise ValueError(f"Unknown integral type: {itype}")
        rkbT, ns, ksl = self.get_rkb_t(k, itype)
        ksr = rkbT.shape[1]
        near = np.zeros((ksl, ksr, ns, ksl + ksr - 1))
        for ip in range(ksl):
            for jp in range(ksr):
                for i in range(ns):
                    first = i + ip - ksl + 1
                    lo, hi = max(0, first), min(ns, i + ksr - jp)
                    if hi > lo:
                        near[ip, jp, i, lo - first:hi - first] = rkbT[ip, jp, i, lo:hi]
        rl, fl = self._pair_moments(k, itype[0])
        rr, fr = self._pair_moments(k, itype[1])
        return near, rl, fl, rr, fr

    def get_symmetric_exchange_factors(self, k, itype="pppp"):
        if itype not in ("pppp", "qqqq"):
            raise ValueError("symmetric exchange factors need equal components")
        near, rising, falling, _, _ = self.get_coulomb_factors(k, itype)
        return near, rising, falling

    def release_shared_banks(self):
        """Drop this grid's device banks for every cache that shares them."""
        with self._lock:
            self._cache.clear()


# ------------------------------------------------------------- densities
def _stack(vectors, ns: int, dev) -> torch.Tensor:
    """Zero-padded (n, ld) device stack of coefficient vectors (ld >= ns, even)."""
    ld = ns + (ns & 1)
    out = np.zeros((len(vectors), ld))
    for r, v in enumerate(vectors):
        v = np.asarray(v, dtype=np.float64).reshape(-1)
        m = min(v.shape[0], ns)
        out[r, :m] = v[:m]
    return torch.from_numpy(out).to(dev)


def cell_densities(bank: CellBank, P: torch.Tensor, Q: torch.Tensor, pairs, nsp: int, nsq: int,
                   stream=None) -> torch.Tensor:
    """D rows [D_P(ab) | D_Q(ab)] (n_pairs, kdim) of the banded pair densities
    of the (a, b) rows of the coefficient stacks P, Q (atomx _density_sym with
    extents nsp and nsq, convol.py:713), in bank index order."""
    L = _native.load()
    pr = torch.as_tensor(np.ascontiguousarray(np.asarray(pairs, dtype=np.int64).reshape(-1, 2)), device=P.device)
    n = int(pr.shape[0])
    D = torch.zeros((max(n, 1), bank.kdim), dtype=torch.float64, device=P.device)
    s = _native.stream_handle(stream)
    ld = P.shape[1]
    for comp, C, nsd, ks, off in (("p", P, nsp, bank.ksp, 0), ("q", Q, nsq, bank.ksq, bank.kp_pad)):
        _native.check(L.rkb_cell_densities(C.data_ptr(), C.data_ptr(), ld, pr.data_ptr(), n, ld, ld,
                                           min(nsd, bank.ns), bank.ns, ks, D.data_ptr(), bank.kdim, off, s),
                      "rkb_cell_densities")
    return D[:n]


def _potentials(bank: CellBank, D: torch.Tensor, stream=None) -> torch.Tensor:
    """W = D K_full^T: row r is the pair potential of density r in bank order."""
    L = _native.load()
    n = D.shape[0]
    W = torch.empty((max(n, 1), bank.kdim), dtype=torch.float64, device=D.device)
    _native.check(L.rkb_gemm_nt_fp64(D.data_ptr(), bank.kdim, bank.K.data_ptr(), bank.kdim, W.data_ptr(), bank.kdim,
                                     n, bank.kdim, bank.kdim, 0, _native.stream_handle(stream)), "rkb_gemm_nt_fp64")
    return W[:n]


def _dots(Dl: torch.Tensor, W: torch.Tensor, il, iw, stream=None) -> torch.Tensor:
    L = _native.load()
    il = torch.as_tensor(np.ascontiguousarray(il, dtype=np.int64), device=Dl.device)
    iw = torch.as_tensor(np.ascontiguousarray(iw, dtype=np.int64), device=Dl.device)
    out = torch.empty(il.shape[0], dtype=torch.float64, device=Dl.device)
    _native.check(L.rkb_cell_dots(Dl.data_ptr(), Dl.shape[1], W.data_ptr(), W.shape[1], Dl.shape[1], il.data_ptr(),
                                  iw.data_ptr(), il.shape[0], out.data_ptr(), _native.stream_handle(stream)),
                  "rkb_cell_dots")
    return out


def _sizes(bd):
    ns = int(bd["ns"])
    return ns, int(bd.get("nsp", ns)), int(bd.get("nsq", ns))


# ------------------------------------------------------ cell integrals
def compute_slater_rk_cell_batch(orbital_arrays, keys, bsp_data, cache=None):
    """R^k(ab, cd) for many (a, b, c, d, k) keys (atomx convol.py:2084).

    ``orbital_arrays`` maps each key to its (P, Q) coefficient vectors.  Per
    multipole: the distinct left pairs (a, b) and right pairs (c, d) become
    banded density rows, the right ones go through one GEMM with the bank
    (their pair potentials), and every integral is one dot.  Returns a list
    aligned with ``keys``.
    """
    _native.require_device()
    cache = cache if isinstance(cache, ConvolCache) else ConvolCache(bsp_data)
    ns, nsp, nsq = _sizes(bsp_data)
    keys = [tuple(kk) for kk in keys]
    if not keys:
        return []
    names = list(dict.fromkeys(x for kk in keys for x in kk[:4]))
    idx = {n: i for i, n in enumerate(names)}
    dev = torch.device("cuda", torch.cuda.current_device())
    P = _stack([orbital_arrays[n][0] for n in names], ns, dev)
    Q = _stack([orbital_arrays[n][1] for n in names], ns, dev)
    result = np.zeros(len(keys))
    by_k: dict = {}
    for e, kk in enumerate(keys):
        by_k.setdefault(int(kk[4]), []).append(e)
    for k, ents in by_k.items():
        bank = cache.bank(k)
        lp = np.array([(idx[keys[e][0]], idx[keys[e][1]]) for e in ents], dtype=np.int64)
        rp = np.array([(idx[keys[e][2]], idx[keys[e][3]]) for e in ents], dtype=np.int64)
        lu, il = np.unique(lp, axis=0, return_inverse=True)
        ru, ir = np.unique(rp, axis=0, return_inverse=True)
        Dl = cell_densities(bank, P, Q, lu, nsp, nsq)
        W = _potentials(bank, cell_densities(bank, P, Q, ru, nsp, nsq))
        result[np.asarray(ents)] = to_host(_dots(Dl, W, il.reshape(-1), ir.reshape(-1)))
    return [float(v) for v in result]


def compute_slater_rk_cell(Pa, Qa, Pb, Qb, Pc, Qc, Pd, Qd, bsp_data, k, cache=None):
    """Scalar cell integral R^k(ab, cd) (atomx convol.py:1756); a non-finite
    value raises FloatingPointError."""
    od = {0: (Pa, Qa), 1: (Pb, Qb), 2: (Pc, Qc), 3: (Pd, Qd)}
    v = compute_slater_rk_cell_batch(od, [(0, 1, 2, 3, int(k))], bsp_data, cache)[0]
    if not np.isfinite(v):
        raise FloatingPointError(f"compute_slater_rk_cell: non-finite R^k (k={k}, value={v})")
    return v


def compute_slater_fk_cell(Pa, Qa, Pb, Qb, bsp_data, k, cache=None):
    """F^k(a, b) = R^k(aa, bb) (convol.py:1885)."""
    return compute_slater_rk_cell(Pa, Qa, Pa, Qa, Pb, Qb, Pb, Qb, bsp_data, k, cache)


def compute_slater_gk_cell(Pa, Qa, Pb, Qb, bsp_data, k, cache=None):
    """G^k(a, b) = R^k(ab, ba) (convol.py:1891)."""
    return compute_slater_rk_cell(Pa, Qa, Pb, Qb, Pb, Qb, Pa, Qa, bsp_data, k, cache)


def cell_tables(P, Q, kappa, bsp_data, k_max: int, cache=None, plan=None, stream=None):
    """Whole cell-engine tables R^k(ac; bd) over every allowed pair (the
    TablePlan of atomx_b200.plan, same layout as the Poisson engine's
    RkTables): per multipole one density block D, one GEMM for the pair
    potentials and one symmetric table contraction."""
    from .plan import make_plan
    from .tables import RkTables, tile_tasks
    L = _native.require_device()
    cache = cache if isinstance(cache, ConvolCache) else ConvolCache(bsp_data)
    plan = plan or make_plan(np.asarray(kappa), k_max)
    ns, nsp, nsq = _sizes(bsp_data)
    dev = torch.device("cuda", torch.cuda.current_device())
    Pd = P if isinstance(P, torch.Tensor) and P.is_cuda else _stack(list(np.asarray(P)), ns, dev)
    Qd = Q if isinstance(Q, torch.Tensor) and Q.is_cuda else _stack(list(np.asarray(Q)), ns, dev)
    sizes = [plan.n_of_k(k) for k in plan.ks]
    offs = np.concatenate([[0], np.cumsum(np.asarray(sizes, dtype=np.int64) ** 2)])
    values = torch.empty(int(offs[-1]), dtype=torch.float64, device=dev)
    s = _native.stream_handle(stream)
    for gi, k in enumerate(plan.ks):
        bank = cache.bank(k, stream)
        D = cell_densities(bank, Pd, Qd, plan.pairs[plan.pairs_of_k[k]], nsp, nsq, stream)
        W = _potentials(bank, D, stream)
        tasks = torch.as_tensor(tile_tasks([sizes[gi]]).reshape(-1), device=dev)
        meta = torch.as_tensor(np.array([0, sizes[gi], int(offs[gi])], dtype=np.int64), device=dev)
        _native.check(L.rkb_table_contract_fp64(D.data_ptr(), W.data_ptr(), bank.kdim, bank.kdim, meta[0:].data_ptr(),
                                                meta[1:].data_ptr(), meta[2:].data_ptr(), tasks.data_ptr(),
                                                tasks.shape[0] // 3, values.data_ptr(), s), "rkb_table_contract_fp64")
    return RkTables(plan=plan, ks=plan.ks, values=values, offsets={k: int(offs[i]) for i, k in enumerate(plan.ks)},
                    precision="cell")


# ------------------------------------------------------------ bilinear
def build_slater_rk_bilinear(Pa, Qa, Pb, Qb, bsp_data, k, cache=None):
    """(M_PP, M_QQ, M_PQ, M_QP) with R^k(a r, b s) = Pr.M_PP.Ps + Qr.M_QQ.Qs
    + Pr.M_PQ.Qs + Qr.M_QP.Ps for any (r, s) (atomx convol.py:1945)."""
    L = _native.require_device()
    cache = cache if isinstance(cache, ConvolCache) else ConvolCache(bsp_data)
    bank = cache.bank(k)
    ns, nsp, nsq = _sizes(bsp_data)
    dev = bank.K.device
    W = _stack([Pa, Qa, Pb, Qb], ns, dev)
    wPa, wQa, wPb, wQb = W[0], W[1], W[2], W[3]
    out = []
    for itype, wa, wb, nl, nr in (("pppp", wPa, wPb, nsp, nsp), ("qqqq", wQa, wQb, nsq, nsq),
                                  ("pqpq", wPa, wQb, min(ns, nsp), min(ns, nsq)),
                                  ("qpqp", wQa, wPb, min(ns, nsq), min(ns, nsp))):
        r0, c0, ksl, ksr = bank.offsets(itype)
        T = torch.empty((ns * nr * ksr,), dtype=torch.float64, device=dev)
        M = torch.empty((ns, ns), dtype=torch.float64, device=dev)
        kb = bank.K[r0:, c0:]
        _native.check(L.rkb_cell_bilinear(kb.data_ptr(), bank.kdim, ns, wa.data_ptr(), wb.data_ptr(), nl, nr, ksl, ksr,
                                          ns, T.data_ptr(), M.data_ptr(), _native.stream_handle()),
                      "rkb_cell_bilinear")
        out.append(M)
    return tuple(to_host(m) for m in out)


def eval_slater_rk_bilinear(M, Pl, Ql, Pr, Qr):
    """One R^k(a l, b r) from the bilinear matrices (convol.py:1981)."""
    M_PP, M_QQ, M_PQ, M_QP = M
    return float(Pl @ (M_PP @ Pr) + Ql @ (M_QQ @ Qr) + Pl @ (M_PQ @ Qr) + Ql @ (M_QP @ Pr))


def compute_slater_rk_table(M, CP_l, CQ_l, CP_r, CQ_r):
    """Table R^k(a l, b r) over coefficient columns (convol.py:1988), as two
    FP64 GEMMs per component block on the device: X = C_l^T M_xy, then
    T += X C_r.  Returns numpy for numpy inputs."""
    L = _native.require_device()
    dev = torch.device("cuda", torch.cuda.current_device())
    host = not any(isinstance(a, torch.Tensor) for a in (CP_l, CQ_l, CP_r, CQ_r))
    Ms = [as_device(m) for m in M]
    ns = Ms[0].shape[0]
    kp = _round16(ns)

    def padded_t(C):  # (n, kp) rows = columns of C, zero padded to kp
        C = as_device(C)
        out = torch.zeros((C.shape[1], kp), dtype=torch.float64, device=dev)
        out[:, :C.shape[0]] = C.t()
        return out

    cl = {"P": padded_t(CP_l), "Q": padded_t(CQ_l)}
    cr = {"P": padded_t(CP_r), "Q": padded_t(CQ_r)}
    nl, nr = cl["P"].shape[0], cr["P"].shape[0]
    T = torch.zeros((nl, nr), dtype=torch.float64, device=dev)
    s = _native.stream_handle()
    for m, a, b in zip(Ms, ("P", "Q", "P", "Q"), ("P", "Q", "Q", "P")):
        mt = torch.zeros((kp, kp), dtype=torch.float64, device=dev)
        mt[:ns, :ns] = m.t()
        X = torch.zeros((nl, kp), dtype=torch.float64, device=dev)   # X = C_l^T M
        _native.check(L.rkb_gemm_nt_fp64(cl[a].data_ptr(), kp, mt.data_ptr(), kp, X.data_ptr(), kp, nl, kp, kp, 0, s),
                      "rkb_gemm_nt_fp64")
        _native.check(L.rkb_gemm_nt_fp64(X.data_ptr(), kp, cr[b].data_ptr(), kp, T.data_ptr(), nr, nl, nr, kp, 1, s),
                      "rkb_gemm_nt_fp64")
    return to_host(T) if host else T


# --------------------------------------------------- direct and exchange
def _full_from_banded(bank: CellBank, Wrow: torch.Tensor, stream=None):
    """(J_PP, J_QQ) device: banded potentials of one W row to full matrices."""
    L = _native.load()
    ns = bank.ns
    out = []
    for off, ks in ((0, bank.ksp), (bank.kp_pad, bank.ksq)):
        V = torch.zeros((ns, ns), dtype=torch.float64, device=Wrow.device)
        v = Wrow[off:off + ks * ns].contiguous()
        _native.check(L.rkb_cell_banded_to_full(v.data_ptr(), ns, ks, 1, V.data_ptr(), _native.stream_handle(stream)),
                      "rkb_cell_banded_to_full")
        out.append(V)
    return out


def compute_direct_potential_cell(orb_P, orb_Q, bsp_data, k, cache=None):
    """Direct matrices (J_PP, J_QQ) of the density P^2 + Q^2, each fed by both
    source components (atomx convol.py:1694)."""
    _native.require_device()
    cache = cache if isinstance(cache, ConvolCache) else ConvolCache(bsp_data)
    bank = cache.bank(k)
    ns = bank.ns
    C = _stack([orb_P, orb_Q], ns, bank.K.device)
    D = cell_densities(bank, C[0:1], C[1:2], [(0, 0)], ns, ns)
    W = _potentials(bank, D)
    return tuple(to_host(m) for m in _full_from_banded(bank, W[0]))


def _exchange_blocks(bank: CellBank, left: dict, right: dict, blocks, symmetric_pairs, stream=None):
    """Device exchange contractions of outer-product densities left[a] x right[b]."""
    L = _native.load()
    ns, dev = bank.ns, bank.K.device
    one = torch.ones(1, dtype=torch.float64, device=dev)
    s = _native.stream_handle(stream)
    out = {}
    for a, b in blocks:
        dens = torch.empty((ns, ns), dtype=torch.float64, device=dev)
        la, rb = left[a].reshape(1, -1), right[b].reshape(1, -1)
        _native.check(L.rkb_cell_exchange_density(la.data_ptr(), rb.data_ptr(), la.shape[1], 1, one.data_ptr(), 1, 1,
                                                  ns, dens.data_ptr(), s), "rkb_cell_exchange_density")
        r0, c0, ksl, ksr = bank.offsets(a + b + a + b)
        kofs = torch.tensor([r0 * bank.kdim + c0], dtype=torch.int64, device=dev)
        res = torch.empty((ns, ns), dtype=torch.float64, device=dev)
        sym = (a, b) in symmetric_pairs
        _native.check(L.rkb_cell_exchange(bank.K.data_ptr(), bank.kdim, kofs.data_ptr(), dens.data_ptr(), 1, ns, ksl,
                                          ksr, int(sym), 0, res.data_ptr(), s), "rkb_cell_exchange")
        out[a, b] = res
    return out


def compute_exchange_matrix_cell(orb_a_P, orb_a_Q, orb_b_P, orb_b_Q, bsp_data, k, cache=None):
    """Exchange blocks (K_PP, K_QQ, K_PQ, K_QP) of the spinor pair density
    (atomx convol.py:1723); with a == b (the same arrays) the equal-component
    blocks are built as symmetric halves and K_QP = K_PQ^T."""
    _native.require_device()
    cache = cache if isinstance(cache, ConvolCache) else ConvolCache(bsp_data)
    bank = cache.bank(k)
    ns = bank.ns
    diagonal = orb_a_P is orb_b_P and orb_a_Q is orb_b_Q
    C = _stack([orb_a_P, orb_a_Q, orb_b_P, orb_b_Q], ns, bank.K.device)
    left, right = {"p": C[0], "q": C[1]}, {"p": C[2], "q": C[3]}
    blocks = [("p", "p"), ("q", "q"), ("p", "q")] + ([] if diagonal else [("q", "p")])
    sym = {("p", "p"), ("q", "q")} if diagonal else set()
    out = _exchange_blocks(bank, left, right, blocks, sym)
    kpp, kqq, kpq = (to_host(out[x]) for x in (("p", "p"), ("q", "q"), ("p", "q")))
    kqp = kpq.T.copy() if diagonal else to_host(out["q", "p"])
    return kpp, kqq, kpq, kqp


# ------------------------------------------------------ DBSR Fock blocks
def build_hf_matrices_dbsr(targets, P_stack, Q_stack, angular_direct, angular_exchange, k_values, norms, bsp_data,
                           cache=None, skip_pq_exchange=False, stream=None):
    """Fock blocks (PP, QQ, PQ, QP) of several target orbitals at once, the
    algorithm of DFSolver._build_hf_matrix_dbsr (methods/dirac_fock.py:1128):
    for each (component block, k) the direct density sum_j a(i,j,k) d(j,j)
    (doubled for j = i) through the bank (case 1) into the PP or QQ block,
    the exchange density sum_j b(i,j,k) P_i x P_j through the exchange
    contraction (case 4) into its block; then symmetrised and divided by the
    target's norm.  P_stack/Q_stack: (n_orb, ns) coefficients;
    angular_*: (n_orb, n_orb, k_max+1); k_values: the multipoles to visit.
    Returns a device tensor (n_targets, 4, ns, ns)."""
    L = _native.require_device()
    cache = cache if isinstance(cache, ConvolCache) else ConvolCache(bsp_data)
    ns = int(bsp_data["ns"])
    dev = torch.device("cuda", torch.cuda.current_device())
    targets = np.asarray(targets, dtype=np.int64).reshape(-1)
    nt = targets.shape[0]
    n_orb = int(np.asarray(P_stack).shape[0])
    P = _stack(list(np.asarray(P_stack)), ns, dev)
    Q = _stack(list(np.asarray(Q_stack)), ns, dev)
    ld = P.shape[1]
    comp = {1: P, 2: Q}
    ad = np.asarray(angular_direct, dtype=np.float64)
    ax = np.asarray(angular_exchange, dtype=np.float64)
    H = torch.zeros((nt, 4, ns, ns), dtype=torch.float64, device=dev)
    s = _native.stream_handle(stream)
    tgt = torch.as_tensor(targets.astype(np.int32), device=dev)
    slot = {(1, 1): 0, (2, 2): 1, (1, 2): 2, (2, 1): 3}
    for ii, jj in ((1, 1), (1, 2), (2, 1), (2, 2)):
        itype = {(1, 1): "pppp", (1, 2): "pqpq", (2, 1): "qpqp", (2, 2): "qqqq"}[ii, jj]
        for k in k_values:
            k = int(k)
            bank = cache.bank(k, stream)
            r0, c0, ks_bra, ks_ket = bank.offsets(itype)
            a = np.ascontiguousarray(ad[targets, :, k])
            b = np.ascontiguousarray(ax[targets, :, k])
            if np.any(a):
                coef = torch.as_tensor(a, device=dev)
                kp = _round16(ks_ket * ns)
                dd = torch.zeros((nt, kp), dtype=torch.float64, device=dev)
                _native.check(L.rkb_cell_direct_density(comp[jj].data_ptr(), ld, n_orb, coef.data_ptr(), n_orb,
                                                        tgt.data_ptr(), nt, ns, ks_ket, dd.data_ptr(), kp, s),
                              "rkb_cell_direct_density")
                v = torch.empty((nt, ks_bra * ns), dtype=torch.float64, device=dev)
                kb = bank.K[r0:r0 + ks_bra * ns, c0:]
                _native.check(L.rkb_gemm_nt_fp64(dd.data_ptr(), kp, kb.data_ptr(), bank.kdim, v.data_ptr(),
                                                 ks_bra * ns, nt, ks_bra * ns, kp, 0, s), "rkb_gemm_nt_fp64")
                tmp = torch.zeros((nt, ns, ns), dtype=torch.float64, device=dev)
                _native.check(L.rkb_cell_banded_to_full(v.data_ptr(), ns, ks_bra, nt, tmp.data_ptr(), s),
                              "rkb_cell_banded_to_full")
                H[:, 0 if ii == 1 else 1] += tmp
            if skip_pq_exchange and ii == 1 and jj == 2:
                continue
            if np.any(b):
                coef = torch.as_tensor(b, device=dev)
                xx = torch.empty((nt, ns, ns), dtype=torch.float64, device=dev)
                _native.check(L.rkb_cell_exchange_density(comp[ii].data_ptr(), comp[jj].data_ptr(), ld, n_orb,
                                                          coef.data_ptr(), n_orb, nt, ns, xx.data_ptr(), s),
                              "rkb_cell_exchange_density")
                kofs = torch.full((nt,), r0 * bank.kdim + c0, dtype=torch.int64, device=dev)
                Kk = torch.empty((nt, ns, ns), dtype=torch.float64, device=dev)
                _native.check(L.rkb_cell_exchange(bank.K.data_ptr(), bank.kdim, kofs.data_ptr(), xx.data_ptr(), nt, ns,
                                                  ks_bra, ks_ket, int(ii == jj), 0, Kk.data_ptr(), s),
                              "rkb_cell_exchange")
                H[:, slot[ii, jj]] += Kk
    out = torch.empty_like(H)
    nrm = torch.as_tensor(np.asarray(norms, dtype=np.float64).reshape(-1), device=dev)
    _native.check(L.rkb_cell_fock_finish(H.data_ptr(), nrm.data_ptr(), ns, int(bool(skip_pq_exchange)), nt,
                                         out.data_ptr(), s), "rkb_cell_fock_finish")
    return out


def build_hf_matrix_dbsr(target_i, P_stack, Q_stack, angular_direct, angular_exchange, k_values, norm_i, bsp_data,
                         cache=None, skip_pq_exchange=False):
    """One target's Fock blocks as numpy (hfm_PP, hfm_QQ, hfm_PQ, hfm_QP)."""
    H = build_hf_matrices_dbsr([target_i], P_stack, Q_stack, angular_direct, angular_exchange, k_values, [norm_i],
                               bsp_data, cache, skip_pq_exchange)
    h = to_host(H[0])
    return h[0], h[1], h[2], h[3]


# --------------------------------------------------- CI pair potentials
def bspline_pair_potential(cache: ConvolCache, ns: int, orders, rank: int, source):
    """The CI cell operator on one explicit banded pair density (atomx
    physics/csf/matrix.py:703 _bspline_pair_potential): source = (d_P (ns,
    ks_p), d_Q (ns, ks_q)); returns the banded potentials (v_P, v_Q), each fed
    by both source components."""
    _native.require_device()
    bank = cache.bank(rank)
    if int(ns) != bank.ns or tuple(int(o) for o in orders) != (bank.ksp, bank.ksq):
        raise ValueError("pair potential sizes do not match the cache's basis")
    D = torch.zeros((1, bank.kdim), dtype=torch.float64, device=bank.K.device)
    for off, ks, d in ((0, bank.ksp, source[0]), (bank.kp_pad, bank.ksq, source[1])):
        D[0, off:off + ks * ns] = as_device(np.asarray(d, dtype=np.float64).T.reshape(-1))
    W = to_host(_potentials(bank, D)[0])
    vp = W[:bank.ksp * ns].reshape(bank.ksp, ns).T.copy()
    vq = W[bank.kp_pad:bank.kp_pad + bank.ksq * ns].reshape(bank.ksq, ns).T.copy()
    return vp, vq


class PairPotentials:
    """Device pair potentials W(k, b, d) of the CI radial evaluator, kept in a
    bounded LRU (atomx physics/csf/matrix.py:723-817 memoises them per
    (rank, b, d)).  ``integrals(keys)`` evaluates many R^k(ac, bd) keys
    (k, a, c, b, d) at once: the missing potentials of the batch in one GEMM
    per rank, then one gathered dot per key."""

    def __init__(self, orbitals: dict, bsp_data, cache: ConvolCache | None = None, capacity: int = 1024):
        if not isinstance(capacity, int) or isinstance(capacity, bool) or capacity < 1:
            raise ValueError("pair potential cache capacity must be a positive integer")
        _native.require_device()
        self.bsp_data, self.capacity = bsp_data, capacity
        self.cache = cache if isinstance(cache, ConvolCache) else ConvolCache(bsp_data)
        self.ns, self.nsp, self.nsq = _sizes(bsp_data)
        self.names = list(orbitals)
        self.index = {n: i for i, n in enumerate(self.names)}
        dev = torch.device("cuda", torch.cuda.current_device())
        self.P = _stack([orbitals[n][0] for n in self.names], self.ns, dev)
        self.Q = _stack([orbitals[n][1] for n in self.names], self.ns, dev)
        self._lru: OrderedDict = OrderedDict()
        self.hits = self.misses = 0

    def _pair(self, x, y):
        i, j = self.index[x], self.index[y]
        return (i, j) if i <= j else (j, i)

    def potentials(self, k: int, pairs) -> torch.Tensor:
        """(n, kdim) device rows W(k, pair) for the given (b, d) pairs."""
        bank = self.cache.bank(k)
        keys = [(int(k),) + self._pair(b, d) for b, d in pairs]
        missing = [kk for kk in dict.fromkeys(keys) if kk not in self._lru]
        self.hits += len(keys) - len(missing)
        self.misses += len(missing)
        if missing:
            D = cell_densities(bank, self.P, self.Q, [kk[1:] for kk in missing], self.nsp, self.nsq)
            W = _potentials(bank, D)
            for r, kk in enumerate(missing):
                self._lru[kk] = W[r]
        rows = []
        for kk in keys:
            self._lru.move_to_end(kk)
            rows.append(self._lru[kk])
        while len(self._lru) > self.capacity:
            self._lru.popitem(last=False)
        return torch.stack(rows) if rows else torch.zeros((0, bank.kdim), dtype=torch.float64, device=bank.K.device)

    def integrals(self, keys) -> np.ndarray:
        """R^k(ac, bd) for keys (k, a, c, b, d): the pair potential of (b, d)
        against the density of (a, c)."""
        out = np.zeros(len(keys))
        by_k: dict = {}
        for e, kk in enumerate(keys):
            by_k.setdefault(int(kk[0]), []).append(e)
        for k, ents in by_k.items():
            bank = self.cache.bank(k)
            W = self.potentials(k, [(keys[e][3], keys[e][4]) for e in ents])
            tgt = [self._pair(keys[e][1], keys[e][2]) for e in ents]
            tu, it = np.unique(np.asarray(tgt, dtype=np.int64).reshape(-1, 2), axis=0, return_inverse=True)
            Dt = cell_densities(bank, self.P, self.Q, tu, self.nsp, self.nsq)
            vals = to_host(_dots(Dt, W.contiguous(), it.reshape(-1), np.arange(len(ents))))
            if not np.all(np.isfinite(vals)):
                raise FloatingPointError("non-finite Slater integral in the batch")
            out[np.asarray(ents)] = vals
        return out


def radial_evaluator(orbitals: dict, bsp_data, pair_potential_cache_size: int | None = None):
    """R^k evaluator for the CI radial keys ("r", k, a, c, b, d) (atomx
    physics/csf/matrix.py:723, the B-spline flavour's Slater branch): a
    callable on one key, with ``.many(keys)`` for batches and
    ``.pair_cache_info()``."""
    pp = PairPotentials(orbitals, bsp_data, capacity=1024 if pair_potential_cache_size is None
                        else pair_potential_cache_size)

    def evaluate(key):
        if key[0] != "r":
            raise ValueError("the device evaluator takes Slater keys ('r', k, a, c, b, d)")
        return float(pp.integrals([key[1:]])[0])

    evaluate.many = lambda keys: pp.integrals([kk[1:] for kk in keys])
    evaluate.pair_cache_info = lambda: {"hits": pp.hits, "misses": pp.misses, "size": len(pp._lru),
                                        "capacity": pp.capacity}
    evaluate.potentials = pp
    return evaluate
