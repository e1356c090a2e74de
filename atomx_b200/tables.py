"""Whole R^k tables of an ion on the device (batched engine).

For an ion (radial basis + spinors) and k_max, ``slater_rk_tables`` returns
every allowed R^k(ac;bd) = sum_i w_i rho_ac(r_i) Y^k[rho_bd](r_i) — the value
atomx's ``slater_rk_poisson`` (numerics/bspline/slater.py:118) gives for each
ordered entry — as one symmetric n_k x n_k table per multipole k over the
pairs that allow k (``TablePlan.pairs_of_k[k]``, kappa-block ordered), in the
shape of atomx's table API (``compute_slater_rk_table``,
numerics/bspline/convol.py:1988).

Precision forms:

* ``"fp64"``  plain engine: orbital values (K1), fused density + Y^k rows
  (K2), FP64 tensor-pipe contraction of the upper table tiles (K3).
* ``"split"`` split engine (see ``atomx_b200.split``): factored Green operator,
  Ozaki-II INT8 residue GEMMs on tcgen05 recombined in FP64.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from functools import lru_cache

import numpy as np
import torch

from . import _native
from .device import as_device, resident
from .plan import TablePlan, make_plan
from .yk import yk_partial_matrices

__all__ = ["IonDevice", "RkTables", "RkStream", "HostTableSink", "HostPackedTables", "PackedShipper", "packed_offsets", "upload_ion", "stage_ion", "evaluate_staged", "upload_values", "slater_rk_tables",
           "slater_rk_tables_from_values", "tables_for", "stream_tables", "iter_blocks", "tile_tasks", "TILE",
           "Fp64Recompute", "fp64_tables_to_host"]

TILE = 128


def _round_up(x: int, m: int) -> int:
    return (x + m - 1) // m * m


@dataclass
class IonDevice:
    """Device-resident inputs of one ion (basis arrays, orbital values, plan)."""
    plan: TablePlan
    nv: int
    ng: int
    n: int
    r: torch.Tensor
    w: torch.Tensor
    mo: torch.Tensor
    mi: torch.Tensor
    Pv: torch.Tensor
    Qv: torch.Tensor
    pairs: torch.Tensor
    row_pair: torch.Tensor
    row_k: torch.Tensor
    extra: dict = field(default_factory=dict)


def upload_ion(ion, k_max: int | None = None, plan: TablePlan | None = None, stream=None) -> IonDevice:
    """Copy an ion's coefficients to the device and evaluate its orbitals (K1)."""
    L = _native.require_device()
    bsp = ion.bsp
    nv, ng = bsp["gr"].shape
    n = nv * ng
    if plan is None:
        plan = make_plan(ion.kappa, ion.spec.k_max if k_max is None else k_max)
    s = _native.stream_handle(stream)
    r = resident(bsp["gr"]).reshape(-1)
    w = resident(bsp["grw"]).reshape(-1)
    mo_h, mi_h = yk_partial_matrices(ng)
    mo, mi = resident(mo_h), resident(mi_h)
    bp, bq = resident(bsp["bsp_p"]), resident(bsp["bsp_q"])
    cp = as_device(ion.P)
    cq = as_device(ion.Q)
    n_orb = cp.shape[0]
    Pv = torch.empty((n_orb, n), device=cp.device, dtype=torch.float64)
    Qv = torch.empty_like(Pv)
    _native.check(L.rkb_eval_orbitals(cp.data_ptr(), cp.shape[1], n_orb, bp.data_ptr(), nv, ng, bsp["ksp"],
                                      bsp["nsp"], Pv.data_ptr(), n, s), "rkb_eval_orbitals(P)")
    _native.check(L.rkb_eval_orbitals(cq.data_ptr(), cq.shape[1], n_orb, bq.data_ptr(), nv, ng, bsp["ksq"],
                                      bsp["nsq"], Qv.data_ptr(), n, s), "rkb_eval_orbitals(Q)")
    pairs, row_pair, row_k = _plan_arrays(plan)
    return IonDevice(plan=plan, nv=nv, ng=ng, n=n, r=r, w=w, mo=mo, mi=mi, Pv=Pv, Qv=Qv,
                     pairs=pairs, row_pair=row_pair, row_k=row_k,
                     extra={"r_host": np.asarray(bsp["gr"], dtype=np.float64).reshape(-1)})


_STAGE_ALIGN = 256


def evaluate_staged(dev: IonDevice, stream) -> None:
    """Evaluate the orbital values (K1) of an ion staged with
    ``stage_ion(..., evaluate=False)`` on ``stream`` (once; later calls do
    nothing)."""
    pending = dev.extra.pop("pending_eval", None)
    if pending is None:
        return
    L = _native.require_device()
    cp, cq, bp, bq, ksp, nsp, ksq, nsq = pending
    h = _native.stream_handle(stream)
    n_orb = dev.Pv.shape[0]
    _native.check(L.rkb_eval_orbitals(cp.data_ptr(), cp.shape[1], n_orb, bp.data_ptr(), dev.nv, dev.ng, ksp, nsp,
                                      dev.Pv.data_ptr(), dev.n, h), "rkb_eval_orbitals(P)")
    _native.check(L.rkb_eval_orbitals(cq.data_ptr(), cq.shape[1], n_orb, bq.data_ptr(), dev.nv, dev.ng, ksq, nsq,
                                      dev.Qv.data_ptr(), dev.n, h), "rkb_eval_orbitals(Q)")


def stage_ion(ion, plan: TablePlan, stream, pinned=None, factor_tables: dict | None = None, evaluate: bool = True):
    """Device inputs of one ion in ONE device allocation and ONE host-to-device
    copy, for callers that prepare many ions with new grids (a serving
    planner): the grid, weights, partial matrices, B-spline values,
    coefficients and plan arrays (and, with ``factor_tables`` =
    split.host_tables(...), the split engine's factor tables and Z counts)
    are packed into the pinned host buffer ``pinned`` (a uint8 CPU tensor;
    grown and returned when too small), copied on ``stream``, and the
    orbital values (K1) are evaluated into the same allocation.  With
    ``evaluate=False`` only the copy is queued (copy engines, no SM time)
    and ``evaluate_staged`` runs K1 later, on the stream that uses the ion.

    Returns (IonDevice, device factor tables or None, pinned buffer).  The
    pinned buffer may be reused once ``stream`` has passed the copy.  Every
    array equals what ``upload_ion`` gives."""
    _native.require_device()
    bsp = ion.bsp
    nv, ng = bsp["gr"].shape
    n = nv * ng
    mo_h, mi_h = yk_partial_matrices(ng)
    parts = [("r", np.asarray(bsp["gr"], dtype=np.float64).reshape(-1)),
             ("w", np.asarray(bsp["grw"], dtype=np.float64).reshape(-1)),
             ("mo", np.asarray(mo_h, dtype=np.float64)), ("mi", np.asarray(mi_h, dtype=np.float64)),
             ("bp", np.asarray(bsp["bsp_p"], dtype=np.float64)), ("bq", np.asarray(bsp["bsp_q"], dtype=np.float64)),
             ("cp", np.asarray(ion.P, dtype=np.float64)), ("cq", np.asarray(ion.Q, dtype=np.float64)),
             ("pairs", plan.pairs.reshape(-1).astype(np.int64, copy=False)),
             ("row_pair", plan.row_pair.astype(np.int64, copy=False)),
             ("row_k", plan.row_k.astype(np.int32))]
    if factor_tables is not None:
        H = factor_tables
        zc = np.zeros(max(plan.ks) + 1, dtype=np.int32)
        for k in plan.ks:
            zc[k] = H["nz"][k]
        parts += [("flat", H["flat"]), ("koff", H["koff"]), ("flat_t", H["flat_t"]), ("koff_t", H["koff_t"]),
                  ("zcount", zc)]
    offs, pos = [], 0
    for _, a in parts:
        offs.append(pos)
        pos += -(-a.nbytes // _STAGE_ALIGN) * _STAGE_ALIGN
    n_in = pos
    n_orb = int(ion.P.shape[0])
    out_off = pos
    pos += 2 * n_orb * n * 8
    if pinned is None or pinned.numel() < n_in:
        pinned = torch.empty(max(n_in, 1 << 20), dtype=torch.uint8, pin_memory=True)
    hb = pinned.numpy()
    for (_, a), o in zip(parts, offs):
        hb[o:o + a.nbytes].view(a.dtype)[:] = a.reshape(-1)
    s = stream if stream is not None else torch.cuda.current_stream()
    with torch.cuda.stream(s):
        buf = torch.empty(pos, dtype=torch.uint8, device=torch.device("cuda", torch.cuda.current_device()))
        buf[:n_in].copy_(pinned[:n_in], non_blocking=True)
    tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.int64): torch.int64, np.dtype(np.int32): torch.int32}
    v = {name: buf[o:o + a.nbytes].view(tdt[a.dtype]).view(a.shape)
         for (name, a), o in zip(parts, offs)}
    Pv = buf[out_off:out_off + n_orb * n * 8].view(torch.float64).view(n_orb, n)
    Qv = buf[out_off + n_orb * n * 8:pos].view(torch.float64).view(n_orb, n)
    dev = IonDevice(plan=plan, nv=nv, ng=ng, n=n, r=v["r"], w=v["w"], mo=v["mo"], mi=v["mi"], Pv=Pv, Qv=Qv,
                    pairs=v["pairs"], row_pair=v["row_pair"], row_k=v["row_k"],
                    extra={"r_host": parts[0][1],
                           "pending_eval": (v["cp"], v["cq"], v["bp"], v["bq"], bsp["ksp"], bsp["nsp"], bsp["ksq"],
                                            bsp["nsq"])})
    if evaluate:
        evaluate_staged(dev, s)
    tables = None
    if factor_tables is not None:
        tables = {k: v[k] for k in ("flat", "koff", "flat_t", "koff_t", "zcount")}
    return dev, tables, pinned


def _plan_arrays(plan: TablePlan):
    """Device copies of a plan's pair and row arrays, kept with the (cached,
    read-only) plan object per device."""
    key = str(torch.device("cuda", torch.cuda.current_device()))
    cache = plan.__dict__.setdefault("_device", {})
    hit = cache.get(key)
    if hit is None:
        dev = torch.device(key)
        # (the plan's arrays are read-only; torch wants writable sources)
        hit = (torch.from_numpy(plan.pairs.reshape(-1).copy()).to(dev),
               torch.from_numpy(plan.row_pair.copy()).to(dev),
               torch.from_numpy(plan.row_k.astype(np.int32)).to(dev))
        hit = cache.setdefault(key, hit)
    return hit


def upload_values(Pv, Qv, kappa, gr, grw, k_max: int, plan: TablePlan | None = None) -> IonDevice:
    """Device inputs from orbital values already on the grid (rows of Pv, Qv
    are P_a(r_i), Q_a(r_i) on the (nv, ng) Gauss grid ``gr``/``grw``)."""
    _native.require_device()
    gr = np.asarray(gr) if not isinstance(gr, torch.Tensor) else gr
    nv, ng = tuple(gr.shape)
    n = nv * ng
    if plan is None:
        plan = make_plan(np.asarray(kappa), k_max)
    mo_h, mi_h = yk_partial_matrices(ng)
    Pd = as_device(Pv).reshape(-1, n).contiguous()
    Qd = as_device(Qv).reshape(-1, n).contiguous()
    pairs, row_pair, row_k = _plan_arrays(plan)
    return IonDevice(plan=plan, nv=nv, ng=ng, n=n, r=resident(gr).reshape(-1), w=resident(grw).reshape(-1),
                     mo=resident(mo_h), mi=resident(mi_h), Pv=Pd, Qv=Qd,
                     pairs=pairs, row_pair=row_pair, row_k=row_k,
                     extra={"r_host": None if isinstance(gr, torch.Tensor) else np.asarray(gr, dtype=np.float64).reshape(-1)})


@lru_cache(maxsize=512)
def _triangle(nt: int) -> np.ndarray:
    """(2, nt (nt + 1) / 2) int32: the row-major upper triangle of nt x nt tiles."""
    t = np.stack(np.triu_indices(nt)).astype(np.int32)
    t.setflags(write=False)
    return t


def tile_tasks(sizes, tile: int = TILE, order=None, block: int | None = None):
    """Upper-triangle tile list [(group, ti, tj)] for groups of the given sizes:
    each group's tiles row-major, groups in order (or in the group order
    ``order``, a permutation of the group indices).

    ``block``: each group's tiles in blocks of block x block tiles instead
    (blocks row-major, tiles row-major inside a block).  Persistent CTAs take
    consecutive tasks, so the tiles in flight at one time then read a few
    row and column panels that stay in L2, where row-major order sweeps a
    whole tile row of column panels (more than L2 holds on large tables)."""
    if block is not None:
        base = tile_tasks(sizes, tile, order)
        if base.shape[0] == 0:
            return base
        g, ti, tj = base[:, 0], base[:, 1], base[:, 2]
        grank = np.concatenate([[0], np.cumsum(g[1:] != g[:-1])])  # groups are contiguous
        return base[np.lexsort((tj, ti, tj // block, ti // block, grank))]
    nt = (np.asarray(sizes, dtype=np.int64).reshape(-1) + tile - 1) // tile
    groups = np.arange(nt.shape[0]) if order is None else np.asarray(order, dtype=np.int64)
    groups = groups[nt[groups] > 0]
    if groups.shape[0] == 0:
        return np.zeros((0, 3), dtype=np.int32)
    tri = [_triangle(int(n)) for n in nt[groups]]
    g = np.repeat(groups.astype(np.int32), [t.shape[1] for t in tri])
    tt = np.concatenate(tri, axis=1)
    return np.stack([g, tt[0], tt[1]], axis=1)


@dataclass
class RkTables:
    """Symmetric R^k tables of one ion: ``table(k)`` is (n_k, n_k)."""
    plan: TablePlan
    ks: list
    values: torch.Tensor          # concatenated row-major tables
    offsets: dict                 # k -> start in ``values``
    precision: str
    info: dict = field(default_factory=dict)

    def table(self, k: int) -> torch.Tensor:
        nk = self.plan.n_of_k(k)
        o = self.offsets[k]
        return self.values[o:o + nk * nk].view(nk, nk)

    def entry(self, k: int, ac: tuple, bd: tuple) -> float:
        """R^k(ac;bd) by orbital indices (a <= c and b <= d not required)."""
        pk = self.plan.pairs_of_k[k]
        pos = {tuple(self.plan.pairs[p]): i for i, p in enumerate(pk)}
        i = pos[tuple(sorted(ac))]
        j = pos[tuple(sorted(bd))]
        return float(self.table(k)[i, j].item())

    def block(self, k: int, block_ac: int, block_bd: int) -> torch.Tensor:
        """The (k, kappa-block_ac, kappa-block_bd) tile of the k-th table."""
        ranges = {b: (s, e) for b, s, e in self.plan.block_ranges_of_k(k)}
        (s1, e1), (s2, e2) = ranges[block_ac], ranges[block_bd]
        return self.table(k)[s1:e1, s2:e2]

    @property
    def ordered_entries(self) -> int:
        return self.plan.ordered_entries


def packed_offsets(plan: TablePlan) -> dict:
    """k -> start of the k-th table in the packed (upper-triangle) layout."""
    offs, pos = {}, 0
    for k in plan.ks:
        n = plan.n_of_k(k)
        offs[k] = pos
        pos += n * (n + 1) // 2
    return offs


@dataclass
class HostPackedTables:
    """R^k tables in pinned host memory, each stored once as its packed upper
    triangle (the table is symmetric: R^k(ac;bd) = R^k(bd;ac)), so the
    device-to-host copy carries every ordered entry in half the bytes.
    ``table(k)`` expands one table; ``entry`` reads one value."""
    plan: TablePlan
    ks: list
    values: torch.Tensor          # CPU (pinned), unique entries of every table
    offsets: dict                 # k -> start in ``values`` (packed_offsets)
    precision: str
    info: dict = field(default_factory=dict)

    def packed(self, k: int) -> np.ndarray:
        n = self.plan.n_of_k(k)
        o = self.offsets[k]
        return self.values[o:o + n * (n + 1) // 2].numpy()

    def table(self, k: int) -> np.ndarray:
        n = self.plan.n_of_k(k)
        iu = np.triu_indices(n)
        full = np.empty((n, n))
        v = self.packed(k)
        full[iu] = v
        full[(iu[1], iu[0])] = v
        return full

    def entry(self, k: int, ac: tuple, bd: tuple) -> float:
        pk = self.plan.pairs_of_k[k]
        pos = {tuple(self.plan.pairs[p]): i for i, p in enumerate(pk)}
        i, j = sorted((pos[tuple(sorted(ac))], pos[tuple(sorted(bd))]))
        n = self.plan.n_of_k(k)
        return float(self.values[self.offsets[k] + i * n - i * (i - 1) // 2 + (j - i)])

    @property
    def ordered_entries(self) -> int:
        return self.plan.ordered_entries

    @property
    def unique_entries(self) -> int:
        return self.plan.unique_entries


class PackedShipper:
    """Ships finished tables to a pinned host buffer in packed form: each
    table is packed on the compute stream into one of two rotating device
    buffers and copied on the copy stream while the next table is computed."""

    def __init__(self, plan: TablePlan, host: torch.Tensor, device, copy_stream):
        self.plan, self.host, self.cs = plan, host, copy_stream
        self.offsets = packed_offsets(plan)
        nmax = max((plan.n_of_k(k) * (plan.n_of_k(k) + 1) // 2 for k in plan.ks), default=1)
        self.bufs = [torch.empty(nmax, dtype=torch.float64, device=device) for _ in range(2)]
        self.free = [None, None]
        self.i = 0

    def ship(self, k: int, table_ptr: int, stream) -> None:
        L = _native.load()
        b = self.i % 2
        self.i += 1
        if self.free[b] is not None:
            stream.wait_event(self.free[b])
        n = self.plan.n_of_k(k)
        m = n * (n + 1) // 2
        _native.check(L.rkb_pack_upper(table_ptr, n, self.bufs[b].data_ptr(), _native.stream_handle(stream)),
                      "rkb_pack_upper")
        ev = torch.cuda.Event()
        ev.record(stream)
        self.cs.wait_event(ev)
        o = self.offsets[k]
        with torch.cuda.stream(self.cs):
            self.host[o:o + m].copy_(self.bufs[b][:m], non_blocking=True)
            fe = torch.cuda.Event()
            fe.record(self.cs)
        self.free[b] = fe


class Fp64Workspace:
    """Device buffers of the plain engine for one ion, reusable across calls."""

    def __init__(self, dev: IonDevice):
        plan = dev.plan
        self.ld = _round_up(dev.n, 32)
        self.g = torch.empty((plan.n_rows, self.ld), device=dev.Pv.device, dtype=torch.float64)
        self.y = torch.empty_like(self.g)
        sizes = [plan.n_of_k(k) for k in plan.ks]
        self.row0 = torch.as_tensor(np.array([plan.k_row_offset[k] for k in plan.ks], dtype=np.int64),
                                    device=self.g.device)
        self.nk = torch.as_tensor(np.array(sizes, dtype=np.int64), device=self.g.device)
        offs = np.concatenate([[0], np.cumsum(np.array(sizes, dtype=np.int64) ** 2)])
        self.out_off = torch.as_tensor(offs[:-1].astype(np.int64), device=self.g.device)
        self.offsets = {k: int(offs[i]) for i, k in enumerate(plan.ks)}
        self.total = int(offs[-1])
        tasks = tile_tasks(sizes)
        self.n_tasks = int(tasks.shape[0])
        self.tasks = torch.as_tensor(tasks.reshape(-1), device=self.g.device)
        bounds = np.searchsorted(tasks[:, 0], np.arange(len(sizes) + 1))
        self.task_range = [(int(bounds[i]), int(bounds[i + 1])) for i in range(len(sizes))]


def run_fp64(dev: IonDevice, ws: Fp64Workspace, out: torch.Tensor, stream=None) -> None:
    """Plain FP64 engine: K2 (density + Y^k rows) then K3 (table contraction)."""
    L = _native.load()
    s = _native.stream_handle(stream)
    plan = dev.plan
    _native.check(L.rkb_table_rows_fp64(dev.Pv.data_ptr(), dev.Qv.data_ptr(), dev.n, dev.pairs.data_ptr(),
                                        dev.row_pair.data_ptr(), dev.row_k.data_ptr(), plan.n_rows,
                                        dev.r.data_ptr(), dev.w.data_ptr(), dev.nv, dev.ng, dev.mo.data_ptr(),
                                        dev.mi.data_ptr(), ws.g.data_ptr(), ws.y.data_ptr(), ws.ld, s),
                  "rkb_table_rows_fp64")
    _native.check(L.rkb_table_contract_fp64(ws.g.data_ptr(), ws.y.data_ptr(), ws.ld, ws.ld, ws.row0.data_ptr(),
                                            ws.nk.data_ptr(), ws.out_off.data_ptr(), ws.tasks.data_ptr(),
                                            ws.n_tasks, out.data_ptr(), s), "rkb_table_contract_fp64")


class Fp64Recompute:
    """Plain FP64 tables for a set of (ion, k) groups, written at given
    offsets of an output buffer: one Y^k-rows launch per group into a shared
    workspace, then one grouped persistent contraction over all of them.
    The split engines use it for the tables whose certificate fails; the plan
    (workspace, group and task lists) is built once and reused."""

    def __init__(self, items):
        """items: [(IonDevice, k, output offset in doubles)]."""
        from .batch import batch_tasks
        self.items = list(items)
        d = self.items[0][0].Pv.device
        self.ld = _round_up(max(dev.n for dev, _, _ in self.items), 32)
        sizes = [dev.plan.n_of_k(k) for dev, k, _ in self.items]
        kdims = [_round_up(dev.n, 16) for dev, _, _ in self.items]
        self.row0 = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.max_kdim = max(kdims)
        self.g = torch.empty((max(int(self.row0[-1]), 1), self.ld), dtype=torch.float64, device=d)
        self.y = torch.empty_like(self.g)
        meta = np.stack([self.row0[:-1], np.asarray(sizes, dtype=np.int64), np.asarray(kdims, dtype=np.int64),
                         np.asarray([o for _, _, o in self.items], dtype=np.int64)])
        self.meta = torch.as_tensor(meta, device=d)
        tasks = batch_tasks(sizes, kdims, "lpt")
        self.n_tasks = int(tasks.shape[0])
        self.tasks = torch.as_tensor(tasks.reshape(-1), device=d)

    def run(self, out: torch.Tensor, stream=None) -> None:
        L = _native.load()
        s = _native.stream_handle(stream)
        for j, (dev, k, _) in enumerate(self.items):
            r0 = int(dev.plan.k_row_offset[k])
            off = int(self.row0[j]) * self.ld * 8
            _native.check(L.rkb_table_rows_fp64(dev.Pv.data_ptr(), dev.Qv.data_ptr(), dev.n, dev.pairs.data_ptr(),
                                                dev.row_pair.data_ptr() + 8 * r0, dev.row_k.data_ptr() + 4 * r0,
                                                dev.plan.n_of_k(k), dev.r.data_ptr(), dev.w.data_ptr(), dev.nv,
                                                dev.ng, dev.mo.data_ptr(), dev.mi.data_ptr(),
                                                self.g.data_ptr() + off, self.y.data_ptr() + off, self.ld, s),
                          "rkb_table_rows_fp64")
        m = self.meta
        _native.check(L.rkb_table_contract_fp64_groups(self.g.data_ptr(), self.y.data_ptr(), self.ld, self.max_kdim,
                                                       m[2].data_ptr(), m[0].data_ptr(), m[1].data_ptr(),
                                                       m[3].data_ptr(), self.tasks.data_ptr(), self.n_tasks,
                                                       out.data_ptr(), s), "rkb_table_contract_fp64_groups")


def fp64_tables_to_host(dev: IonDevice, ws: Fp64Workspace, out: torch.Tensor, host: torch.Tensor, stream=None,
                        copy_stream=None, packed: bool = False) -> None:
    """Plain FP64 engine with each multipole's table copied to ``host`` on
    ``copy_stream`` while the next one is contracted (``packed``: each
    table's upper triangle, at packed_offsets); returns when done."""
    L = _native.load()
    s = stream if stream is not None else torch.cuda.current_stream()
    cs = copy_stream if copy_stream is not None else torch.cuda.Stream(device=out.device)
    h = _native.stream_handle(s)
    plan = dev.plan
    _native.check(L.rkb_table_rows_fp64(dev.Pv.data_ptr(), dev.Qv.data_ptr(), dev.n, dev.pairs.data_ptr(),
                                        dev.row_pair.data_ptr(), dev.row_k.data_ptr(), plan.n_rows,
                                        dev.r.data_ptr(), dev.w.data_ptr(), dev.nv, dev.ng, dev.mo.data_ptr(),
                                        dev.mi.data_ptr(), ws.g.data_ptr(), ws.y.data_ptr(), ws.ld, h),
                  "rkb_table_rows_fp64")
    shipper = PackedShipper(plan, host, out.device, cs) if packed else None
    for gi, k in enumerate(plan.ks):
        t0, t1 = ws.task_range[gi]
        nk, o = plan.n_of_k(k), ws.offsets[k]
        _native.check(L.rkb_table_contract_fp64(ws.g.data_ptr(), ws.y.data_ptr(), ws.ld, ws.ld, ws.row0.data_ptr(),
                                                ws.nk.data_ptr(), ws.out_off.data_ptr(), ws.tasks.data_ptr() + 12 * t0,
                                                t1 - t0, out.data_ptr(), h), "rkb_table_contract_fp64")
        if shipper is not None:
            shipper.ship(k, out.data_ptr() + 8 * o, s)
            continue
        ev = torch.cuda.Event()
        ev.record(s)
        cs.wait_event(ev)
        with torch.cuda.stream(cs):
            host[o:o + nk * nk].copy_(out[o:o + nk * nk], non_blocking=True)
    cs.synchronize()


def slater_rk_tables(ion, k_max: int | None = None, precision: str = "fp64", stream=None, sink=None,
                     host: bool = False, packed: bool = False, **split_opts):
    """All R^k tables of one ion on the device (see module docstring).

    With ``sink`` the tables are streamed instead of returned: the engine
    computes one multipole table at a time into one of two rotating device
    buffers and calls ``sink(k, table, blocks, stream)`` with the n_k x n_k
    device view and the table's kappa-block row ranges [(block, start, stop)];
    the view is valid for work the sink enqueues on ``stream`` (or finishes
    before returning).  ``iter_blocks`` splits it into (k, kappa_ac-block,
    kappa_bd-block) tiles; ``HostTableSink`` copies tables to pinned host
    memory.  Returns an ``RkStream`` summary in that case.

    With ``host=True`` the tables come back in pinned host memory
    (``values`` is a CPU tensor): each multipole's table is copied while the
    next one is contracted, so the device-to-host copy hides the compute.
    ``packed=True`` (with ``host=True``) ships each table's upper triangle
    only and returns a ``HostPackedTables``: every ordered entry in half the
    bytes.
    """
    if precision not in ("fp64", "split"):
        raise ValueError(f"unknown precision {precision!r}; choose 'fp64' or 'split'")
    dev = upload_ion(ion, k_max=k_max, stream=stream)
    if sink is not None:
        return stream_tables(dev, sink, precision=precision, stream=stream, **split_opts)
    return tables_for(dev, precision=precision, stream=stream, host=host, packed=packed, **split_opts)


@dataclass
class RkStream:
    """Summary of a streamed table run (the values went to the sink)."""
    plan: TablePlan
    ks: list
    precision: str
    device_bytes: int             # engine buffers held while streaming
    info: dict = field(default_factory=dict)


def iter_blocks(table: torch.Tensor, blocks):
    """(kappa_ac-block, kappa_bd-block, tile view) over one multipole table."""
    for b1, s1, e1 in blocks:
        for b2, s2, e2 in blocks:
            yield b1, b2, table[s1:e1, s2:e2]


class HostTableSink:
    """Sink that copies each multipole table to pinned host memory.

    ``tables[k]`` is valid after ``wait()`` (or ``wait(k)``).  One table is
    kept per multipole: a later delivery of the same k replaces it.
    """

    replaces_tables = True

    def __init__(self):
        self.tables, self._events = {}, {}

    def __call__(self, k, table, blocks, stream):
        host = torch.empty(table.shape, dtype=table.dtype, pin_memory=True)
        with torch.cuda.stream(stream):
            host.copy_(table, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        self.tables[k], self._events[k] = host, ev

    def wait(self, k=None):
        for kk in ([k] if k is not None else list(self._events)):
            self._events[kk].synchronize()
        return self.tables if k is None else self.tables[k]


def stream_tables(dev: IonDevice, sink, precision: str = "fp64", stream=None, **split_opts) -> RkStream:
    """Stream every multipole table of ``dev`` to ``sink`` (see ``slater_rk_tables``)."""
    s = stream if stream is not None else torch.cuda.current_stream()
    plan = dev.plan
    if precision == "split":
        from .split import SplitEngine
        eng = SplitEngine(dev, materialize=False, **split_opts)
        eng.stream_tables(sink, stream=s)
        info = eng.info()
        held = eng.held_bytes
    else:
        L = _native.load()
        ws = Fp64Workspace(dev)
        h = _native.stream_handle(s)
        _native.check(L.rkb_table_rows_fp64(dev.Pv.data_ptr(), dev.Qv.data_ptr(), dev.n, dev.pairs.data_ptr(),
                                            dev.row_pair.data_ptr(), dev.row_k.data_ptr(), plan.n_rows,
                                            dev.r.data_ptr(), dev.w.data_ptr(), dev.nv, dev.ng, dev.mo.data_ptr(),
                                            dev.mi.data_ptr(), ws.g.data_ptr(), ws.y.data_ptr(), ws.ld, h),
                      "rkb_table_rows_fp64")
        nmax = max(plan.n_of_k(k) for k in plan.ks)
        bufs = [torch.empty(nmax * nmax, dtype=torch.float64, device=dev.Pv.device) for _ in range(2)]
        zero = torch.zeros(len(plan.ks), dtype=torch.int64, device=dev.Pv.device)
        held = (ws.g.numel() + ws.y.numel() + 2 * nmax * nmax) * 8
        for gi, k in enumerate(plan.ks):
            nk = plan.n_of_k(k)
            t0, t1 = ws.task_range[gi]
            buf = bufs[gi % 2][:nk * nk]
            _native.check(L.rkb_table_contract_fp64(ws.g.data_ptr(), ws.y.data_ptr(), ws.ld, ws.ld,
                                                    ws.row0.data_ptr(), ws.nk.data_ptr(), zero.data_ptr(),
                                                    ws.tasks.data_ptr() + 12 * t0, t1 - t0, buf.data_ptr(), h),
                          "rkb_table_contract_fp64")
            sink(k, buf.view(nk, nk), plan.block_ranges_of_k(k), s)
        info = {}
    return RkStream(plan=plan, ks=plan.ks, precision=precision, device_bytes=int(held), info=info)


def slater_rk_tables_from_values(Pv, Qv, kappa, gr, grw, k_max: int, precision: str = "fp64", stream=None,
                                 **split_opts) -> RkTables:
    """All R^k tables from orbital values on the grid (no B-spline stage)."""
    if precision not in ("fp64", "split"):
        raise ValueError(f"unknown precision {precision!r}; choose 'fp64' or 'split'")
    dev = upload_values(Pv, Qv, kappa, gr, grw, k_max)
    return tables_for(dev, precision=precision, stream=stream, **split_opts)


def tables_for(dev: IonDevice, precision: str = "fp64", stream=None, host: bool = False, packed: bool = False,
               **split_opts):
    if packed and not host:
        raise ValueError("packed tables are a host format: pass host=True")
    if packed:
        plan = dev.plan
        values = torch.empty(max(plan.unique_entries, 1), dtype=torch.float64, pin_memory=True)
        if precision == "split":
            from .split import SplitEngine
            eng = SplitEngine(dev, **split_opts)
            eng.run_to_host(values, stream=stream, packed=True)
            info = eng.info()
        else:
            ws = Fp64Workspace(dev)
            out = torch.empty(ws.total, device=dev.Pv.device, dtype=torch.float64)
            fp64_tables_to_host(dev, ws, out, values, stream=stream, packed=True)
            info = {}
        return HostPackedTables(plan=plan, ks=plan.ks, values=values, offsets=packed_offsets(plan),
                                precision=precision, info=info)
    if precision == "split":
        from .split import SplitEngine
        eng = SplitEngine(dev, **split_opts)
        if host:
            values = torch.empty(eng.total, dtype=torch.float64, pin_memory=True)
            eng.run_to_host(values, stream=stream)
        else:
            values = eng.run(stream=stream, check=True)
        return RkTables(plan=dev.plan, ks=dev.plan.ks, values=values, offsets=eng.offsets, precision="split",
                        info=eng.info())
    ws = Fp64Workspace(dev)
    out = torch.empty(ws.total, device=dev.Pv.device, dtype=torch.float64)
    if host:
        values = torch.empty(ws.total, dtype=torch.float64, pin_memory=True)
        fp64_tables_to_host(dev, ws, out, values, stream=stream)
    else:
        run_fp64(dev, ws, out, stream=stream)
        values = out
    return RkTables(plan=dev.plan, ks=dev.plan.ks, values=values, offsets=ws.offsets, precision="fp64")
