"""Many ions' R^k tables in one persistent launch, replayed as a CUDA graph.

A batch concatenates the (pair, k) rows of every ion into one row space.
One contraction launch then covers the upper tiles of every (ion, k) table:
persistent CTAs walk a single task list, and each task carries its group's
row offset, size and contraction length. Ions of different grids (N, n_gauss)
and table sizes therefore share the launch. The per-ion row kernels (grids
differ per ion) and the contraction are captured once into a CUDA graph and
replayed.

* ``SplitBatch``: the split engine. Every ion's rows are written into one
  pair of int8 residue matrices through ``split.IonRows``, and one
  ``crt_syrk_kernel`` runs over all (ion, k) groups.
* ``Fp64Batch``: the plain engine. Every ion's g and Y^k rows go into one
  (rows, ld) pair, and one ``fp64tab::contract_kernel`` runs with a
  contraction length per group.

The task order matters for balance: tasks cost in proportion to their
group's contraction length, and persistent CTAs take tasks round-robin.
``order="lpt"`` sorts tasks by decreasing cost (longest first); ``"group"``
keeps the table order. ``atomx_b200.autotune`` picks the order, the split
width (bits, and so the number of moduli) and the row-kernel layout by
timing them on the batch under the error gate.

This has no single atomx counterpart. atomx computes each table with
per-integral ``slater_rk_poisson`` calls (numerics/bspline/slater.py:118) or
``compute_slater_rk_table`` (numerics/bspline/convol.py:1988) per ion.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native
from .split import (CB_STRIDE, CERT_LIMIT, IonRows, _round_up, certify, check_kdim, choose_width, join_stream,
                    read_status)
from .split_plan import crt_constants
from .tables import TILE, Fp64Recompute, IonDevice, RkTables, tile_tasks

__all__ = ["SplitBatch", "Fp64Batch", "Workspace", "batch_tasks"]


def batch_tasks(sizes, costs, order: str = "lpt") -> np.ndarray:
    """Upper-triangle tile tasks (group, ti, tj) of all groups, ordered.

    ``costs[g]`` is the relative cost of one tile of group g (its
    contraction length). "lpt" puts the most expensive tiles first (persistent
    CTAs then finish close together): groups by decreasing cost, ties in
    group order, each group's tiles row-major; "group" keeps groups in order.
    """
    if order == "lpt":
        c = np.asarray(costs, dtype=np.float64).reshape(-1)
        return tile_tasks(sizes, order=np.argsort(-c, kind="stable"))
    if order != "group":
        raise ValueError(f"unknown task order {order!r}")
    return tile_tasks(sizes)


class Workspace:
    """Device memory a caller reuses from one batch to the next (a serving
    slot keeps one): ``take`` carves 256-byte aligned views out of one
    buffer, adding a chunk when a batch needs more than it holds, and
    ``reset`` merges the chunks into one buffer for the next batch.  After a
    few batches the largest one fits and no batch allocates device memory.
    Views taken since the last ``reset`` are valid until the next: reset only
    once the previous batch's work, and every sink's work on its tables, is
    done."""

    ALIGN = 256
    MIN_CHUNK = 64 << 20

    def __init__(self, device=None):
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.chunks: list = []
        self.pos = 0      # offset in the last chunk
        self.taken = 0    # aligned bytes taken since the last reset

    @property
    def capacity(self) -> int:
        return int(sum(c.numel() for c in self.chunks))

    def take(self, shape, dtype) -> torch.Tensor:
        shape = tuple(int(x) for x in (shape if isinstance(shape, (tuple, list)) else (shape,)))
        nbytes = int(np.prod(shape, dtype=np.int64)) * torch.empty((), dtype=dtype).element_size()
        step = -(-nbytes // self.ALIGN) * self.ALIGN
        if not self.chunks or self.pos + step > self.chunks[-1].numel():
            self.chunks.append(torch.empty(max(step, self.MIN_CHUNK), dtype=torch.uint8, device=self.device))
            self.pos = 0
        t = self.chunks[-1][self.pos:self.pos + nbytes].view(dtype).view(shape)
        self.pos += step
        self.taken += step
        return t

    def reserve(self, nbytes: int) -> None:
        """Hold at least ``nbytes`` in one buffer from now on (call between
        batches, with nothing taken)."""
        if self.taken:
            raise RuntimeError("reserve() with views taken; call reset() first")
        if self.capacity < nbytes or len(self.chunks) > 1:
            self.chunks = []
            self.chunks = [torch.empty(max(int(nbytes), self.capacity), dtype=torch.uint8, device=self.device)]
        self.pos = 0

    def reset(self) -> None:
        if len(self.chunks) > 1:
            need = self.taken
            self.chunks = []  # back to the caching allocator before the merged buffer is taken
            self.chunks = [torch.empty(need, dtype=torch.uint8, device=self.device)]
        self.pos = 0
        self.taken = 0


def _alloc(workspace, shape, dtype, device):
    if workspace is None:
        return torch.empty(shape, dtype=dtype, device=device)
    return workspace.take(shape, dtype)


class _Graphable:
    """Shared CUDA-graph capture of ``step()``."""

    graph = None

    def capture(self, stream=None):
        """Record ``step()`` once into a CUDA graph (after one eager warm-up,
        which also performs every one-time attribute set-up)."""
        s = stream if stream is not None else torch.cuda.Stream()
        self.step(s)
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.step(s)
        self.graph = g
        return g

    def replay(self):
        """Replay the captured step on the current stream."""
        if self.graph is None:
            self.capture()
        self._stream = torch.cuda.current_stream()
        self.graph.replay()


class SplitBatch(_Graphable):
    """Split-precision tables of many ions with one contraction launch."""

    dominant_kernel = "split::crt_syrk_kernel"

    def __init__(self, devs: list[IonDevice], bits: int | None = None, tau: float = 1e-3, fused=None,
                 corr_floor: float | None = None, order: str = "lpt", n_mod: int | None = None,
                 cert_limit: float = CERT_LIMIT, ion_widths: bool = False, ion_rows: list | None = None,
                 workspace: Workspace | None = None):
        _native.require_device()
        if not devs:
            raise ValueError("empty batch")
        self.devs, self.order = list(devs), order
        if ion_rows is not None:  # row sides built ahead (e.g. by a serving planner)
            if len(ion_rows) != len(self.devs) or any(r.dev is not d for r, d in zip(ion_rows, self.devs)):
                raise ValueError("ion_rows must be the IonRows of devs, in order")
            self.ions = list(ion_rows)
        else:
            self.ions = [IonRows(d, tau=tau, fused=fused) for d in self.devs]
        d = self.devs[0].Pv.device
        self.kpad = max(r.kmax_dim for r in self.ions)
        check_kdim(self.kpad)
        self.bits, self.n_mod = choose_width(bits, n_mod, self.kpad)
        #: split width of each ion's rows.  With ``ion_widths`` every ion takes
        #: the widest split the batch's moduli hold at its own contraction
        #: length (or ``bits``), so an ion's rows, and with a fixed n_mod and
        #: corr_floor its tables, do not depend on the other ions of the batch.
        self.ion_bits = [choose_width(bits, self.n_mod, r.kmax_dim)[0] if ion_widths else self.bits
                         for r in self.ions]
        self.bits = min(self.ion_bits)
        self.moduli, self.f_hi, self.f_lo, self.M, self.pair_inv = crt_constants(self.n_mod)
        self.cw = max(dv.ng for dv in self.devs) + 2  # g_0 and the two coupling moments
        self.cwp = _round_up(self.cw, 2)
        counts = [dv.plan.n_rows for dv in self.devs]
        self.row_base = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        nrows = int(self.row_base[-1])
        self.rows_alloc = _round_up(max(nrows, 1), TILE)
        ws = workspace
        res_shape = (self.n_mod, self.rows_alloc, self.kpad)
        self.resA = _alloc(ws, res_shape, torch.int8, d)
        self.resB = _alloc(ws, res_shape, torch.int8, d) if any(r.has_z for r in self.ions) else None
        # The cell and two-kernel row paths write every column of their rows;
        # the fused kernel only its own.  Padding rows are read by the last
        # tiles (their entries are never stored) and are zeroed all the same.
        full_zero = any(r.kind == "fused" for r in self.ions)
        for res in (self.resA, self.resB):
            if res is not None:
                (res if full_zero else res[:, nrows:, :]).zero_()
        self.rowscale = _alloc(ws, (nrows,), torch.float64, d)
        # core vectors: an ion writes its own ng + 2 columns of the batch's cwp
        self.left = _alloc(ws, (nrows, self.cwp), torch.float64, d)
        self.right = _alloc(ws, (nrows, self.cwp), torch.float64, d)
        self.left.zero_()
        self.right.zero_()
        self.cbound = _alloc(ws, (nrows, CB_STRIDE), torch.float64, d)
        two = [dv.plan.n_rows for dv, r in zip(self.devs, self.ions) if r.kind == "two"]
        self.xwork = _alloc(ws, (max(two), self.kpad), torch.float64, d) if two else None
        self.corr_floor = 2.0 ** -(self.bits + 10) if corr_floor is None else float(corr_floor)
        # groups: (ion, k)
        g_row0, g_n, g_kdim, self.group_of = [], [], [], []
        for i, (dv, r) in enumerate(zip(self.devs, self.ions)):
            for k in dv.plan.ks:
                g_row0.append(int(self.row_base[i]) + dv.plan.k_row_offset[k])
                g_n.append(dv.plan.n_of_k(k))
                g_kdim.append(r.kdim[k])
                self.group_of.append((i, k))
        offs = np.concatenate([[0], np.cumsum(np.asarray(g_n, dtype=np.int64) ** 2)])
        self.offsets = {gk: int(offs[j]) for j, gk in enumerate(self.group_of)}
        self.total = int(offs[-1])
        tasks = batch_tasks(g_n, g_kdim, order)
        self.n_tasks = int(tasks.shape[0])
        # the group records and the task list in one host-to-device copy
        ng_ = len(g_n)
        host = np.empty(4 * ng_ + (tasks.size + 1) // 2, dtype=np.int64)
        host[:4 * ng_] = np.concatenate([g_row0, g_n, g_kdim, offs[:-1]]).astype(np.int64)
        host[4 * ng_:].view(np.int32)[:tasks.size] = tasks.reshape(-1)
        arr = torch.from_numpy(host).to(d)
        self.grp_row0, self.grp_n, self.grp_kdim, self.grp_out = (arr[i * ng_:(i + 1) * ng_] for i in range(4))
        self.tasks = arr[4 * ng_:].view(torch.int32)[:tasks.size]
        #: [contraction status, number of tables whose certificate failed]
        self.status = torch.zeros(2, dtype=torch.int32, device=d)
        self.est = torch.zeros(len(g_n), dtype=torch.float64, device=d)
        self.cert_limit = float(cert_limit)
        #: (ion, k) tables recomputed in FP64 by the last check_status()
        self.escalated: list = []
        self._stream = None
        self.out = _alloc(ws, (self.total,), torch.float64, d)
        self._c = (np.ctypeslib.as_ctypes(np.ascontiguousarray(self.moduli, dtype=np.int32)),
                   np.ctypeslib.as_ctypes(np.ascontiguousarray(self.f_hi)),
                   np.ctypeslib.as_ctypes(np.ascontiguousarray(self.f_lo)),
                   np.ctypeslib.as_ctypes(np.ascontiguousarray(np.concatenate([self.pair_inv, [1]]).astype(np.int32))))

    @property
    def launches_per_step(self) -> int:
        """Row kernels of every ion, the certificate and the contraction."""
        return sum(2 if r.kind == "two" else 1 for r in self.ions) + 2

    @property
    def ordered_entries(self) -> int:
        return sum(dv.plan.ordered_entries for dv in self.devs)

    #: side streams the per-ion row launches are spread over
    ROW_STREAMS = 4

    def rows(self, stream=None, side_streams=None) -> None:
        """Every ion's row kernels, then the certificate.  Ions on the cell or
        fused kernel go round-robin to side streams (``side_streams``, else
        ROW_STREAMS of the batch's own) forked from and joined back to
        ``stream`` (a fork/join that graph capture records), so small ions
        fill the GPU side by side; two-kernel ions share the FP64 workspace
        and stay in order on ``stream``."""
        s = stream if stream is not None else torch.cuda.current_stream()
        self._stream = stream
        if side_streams is not None:
            self._side = list(side_streams)
        elif not hasattr(self, "_side"):
            self._side = [torch.cuda.Stream(device=s.device) for _ in range(self.ROW_STREAMS)]
        fork = torch.cuda.Event()
        fork.record(s)
        used = set()
        j = 0
        for i, r in enumerate(self.ions):
            if r.kind == "two":
                ls = s
            else:
                ls = self._side[j % len(self._side)]
                j += 1
                if ls not in used:
                    ls.wait_event(fork)
                    used.add(ls)
            r.launch(self.ion_bits[i], self.n_mod, self._c[0], self.resA, self.resB, self.kpad, int(self.row_base[i]),
                     self.rows_alloc, self.rowscale, self.left, self.right, self.cbound, self.cwp, self.xwork, ls)
        for ls in used:
            join = torch.cuda.Event()
            join.record(ls)
            s.wait_event(join)
        certify(self.grp_row0, self.grp_n, self.rowscale, self.cbound, self.cert_limit, self.est, self.status, s)

    def contract(self, stream=None) -> None:
        L = _native.load()
        _native.check(L.rkb_split_contract(self.resA.data_ptr(), _native.ptr(self.resB), self.kpad, self.rows_alloc,
                                           self.n_mod, self._c[0], self._c[3], self._c[1], self._c[2], self.M,
                                           self.rowscale.data_ptr(), self.left.data_ptr(), self.right.data_ptr(),
                                           self.cbound.data_ptr(), self.corr_floor, self.cw, self.cwp,
                                           self.grp_row0.data_ptr(), self.grp_n.data_ptr(),
                                           self.grp_kdim.data_ptr(), self.grp_out.data_ptr(), self.tasks.data_ptr(),
                                           self.n_tasks, self.out.data_ptr(), self.status.data_ptr(),
                                           _native.stream_handle(stream)),
                      "rkb_split_contract")

    def step(self, stream=None, side_streams=None) -> None:
        """Enqueue every row launch and the one contraction (no host sync)."""
        self.rows(stream, side_streams)
        self.contract(stream)

    def check_status(self) -> None:
        """Wait for the device, raise a contraction error, and recompute in FP64
        every (ion, k) table whose certificate failed (listed in ``escalated``)."""
        s, (st, flagged) = read_status(self.status, self._stream)
        if st:
            self.status[0] = 0
            _native.check(st, "crt_syrk_kernel")
        self.escalated = []
        if flagged:
            est = self.est.cpu().numpy()
            self.escalated = [gk for j, gk in enumerate(self.group_of) if not est[j] <= self.cert_limit]
            key = tuple(self.escalated)
            cache = self.__dict__.setdefault("_recompute_cache", {})
            if key not in cache:
                cache[key] = Fp64Recompute([(self.devs[i], k, self.offsets[(i, k)]) for i, k in key])
            cache[key].run(self.out, s)
            join_stream(s)

    def table(self, ion: int, k: int) -> torch.Tensor:
        nk = self.devs[ion].plan.n_of_k(k)
        o = self.offsets[(ion, k)]
        return self.out[o:o + nk * nk].view(nk, nk)

    def tables(self, ion: int) -> RkTables:
        plan = self.devs[ion].plan
        o0 = self.offsets[(ion, plan.ks[0])]
        n = sum(plan.n_of_k(k) ** 2 for k in plan.ks)
        return RkTables(plan=plan, ks=plan.ks, values=self.out[o0:o0 + n],
                        offsets={k: self.offsets[(ion, k)] - o0 for k in plan.ks}, precision="split",
                        info={"bits": self.bits, "n_mod": self.n_mod, "fused": self.ions[ion].fused})

    def info(self) -> dict:
        return {"ions": len(self.devs), "bits": self.bits, "ion_bits": sorted(set(self.ion_bits)),
                "n_mod": self.n_mod, "kpad": self.kpad,
                "order": self.order, "tasks": self.n_tasks, "rows": int(self.row_base[-1]),
                "cert_limit": self.cert_limit, "fp64_tables": [list(t) for t in self.escalated],
                "row_kernels": {kd: sum(r.kind == kd for r in self.ions) for kd in ("cells", "fused", "two")},
                "entries": self.ordered_entries}


class Fp64Batch(_Graphable):
    """Plain FP64 tables of many ions with one contraction launch."""

    dominant_kernel = "fp64tab::contract_kernel"

    def __init__(self, devs: list[IonDevice], order: str = "lpt", workspace: Workspace | None = None):
        _native.require_device()
        if not devs:
            raise ValueError("empty batch")
        self.devs, self.order = list(devs), order
        d = self.devs[0].Pv.device
        self.ld = _round_up(max(dv.n for dv in self.devs), 32)
        counts = [dv.plan.n_rows for dv in self.devs]
        self.row_base = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        nrows = int(self.row_base[-1])
        self.g = _alloc(workspace, (nrows, self.ld), torch.float64, d)
        self.y = _alloc(workspace, (nrows, self.ld), torch.float64, d)
        g_row0, g_n, g_kdim, self.group_of = [], [], [], []
        for i, dv in enumerate(self.devs):
            for k in dv.plan.ks:
                g_row0.append(int(self.row_base[i]) + dv.plan.k_row_offset[k])
                g_n.append(dv.plan.n_of_k(k))
                g_kdim.append(_round_up(dv.n, 16))
                self.group_of.append((i, k))
        self.max_kdim = max(g_kdim)
        offs = np.concatenate([[0], np.cumsum(np.asarray(g_n, dtype=np.int64) ** 2)])
        self.offsets = {gk: int(offs[j]) for j, gk in enumerate(self.group_of)}
        self.total = int(offs[-1])
        self.grp_row0 = torch.as_tensor(g_row0, dtype=torch.int64, device=d)
        self.grp_n = torch.as_tensor(g_n, dtype=torch.int64, device=d)
        self.grp_kdim = torch.as_tensor(g_kdim, dtype=torch.int64, device=d)
        self.grp_out = torch.as_tensor(offs[:-1], dtype=torch.int64, device=d)
        tasks = batch_tasks(g_n, g_kdim, order)
        self.n_tasks = int(tasks.shape[0])
        self.tasks = torch.as_tensor(tasks.reshape(-1), device=d)
        self.out = _alloc(workspace, (self.total,), torch.float64, d)

    @property
    def launches_per_step(self) -> int:
        return len(self.devs) + 1

    @property
    def ordered_entries(self) -> int:
        return sum(dv.plan.ordered_entries for dv in self.devs)

    def step(self, stream=None) -> None:
        L = _native.load()
        h = _native.stream_handle(stream)
        for i, dv in enumerate(self.devs):
            off = int(self.row_base[i]) * self.ld * 8
            _native.check(L.rkb_table_rows_fp64(dv.Pv.data_ptr(), dv.Qv.data_ptr(), dv.n, dv.pairs.data_ptr(),
                                                dv.row_pair.data_ptr(), dv.row_k.data_ptr(), dv.plan.n_rows,
                                                dv.r.data_ptr(), dv.w.data_ptr(), dv.nv, dv.ng, dv.mo.data_ptr(),
                                                dv.mi.data_ptr(), self.g.data_ptr() + off, self.y.data_ptr() + off,
                                                self.ld, h),
                          "rkb_table_rows_fp64")
        _native.check(L.rkb_table_contract_fp64_groups(self.g.data_ptr(), self.y.data_ptr(), self.ld, self.max_kdim,
                                                       self.grp_kdim.data_ptr(), self.grp_row0.data_ptr(),
                                                       self.grp_n.data_ptr(), self.grp_out.data_ptr(),
                                                       self.tasks.data_ptr(), self.n_tasks, self.out.data_ptr(), h),
                      "rkb_table_contract_fp64_groups")

    def check_status(self) -> None:
        return None

    def table(self, ion: int, k: int) -> torch.Tensor:
        nk = self.devs[ion].plan.n_of_k(k)
        o = self.offsets[(ion, k)]
        return self.out[o:o + nk * nk].view(nk, nk)

    def info(self) -> dict:
        return {"ions": len(self.devs), "ld": self.ld, "order": self.order, "tasks": self.n_tasks,
                "rows": int(self.row_base[-1]), "entries": self.ordered_entries}
