"""Split-precision R^k engine (host orchestration of K2x + K3s).

For one ion on the device this builds, once per radial grid, the factored
Green operator of every multipole (``split_plan.green_factor``), then per
call runs

* K2x ``rkb_split_rows``: one warp per (pair, k) row forms rho, the factored
  row [X | Z] and its FP64 core correction vectors, scales the row by a power
  of two to ``bits`` bits and writes int8 residues for every CRT modulus;
* K3s ``rkb_split_contract``: per multipole, the upper 128x128 tiles of the
  table as n_mod INT8 GEMMs on tcgen05 with int32 accumulators in TMEM,
  recombined in FP64 by the Chinese remainder theorem, scaled back and
  corrected by the FP64 core terms; tiles above the diagonal are also stored
  transposed.

``bits`` sets the fixed-point width of the split (error about 2^-bits of the
Schwarz scale sqrt(R_acac R_bdbd) of each entry); the number of moduli follows
from ``bits`` and the contraction length.
"""
from __future__ import annotations

import hashlib
import threading

import numpy as np
import torch

from . import _native
from .split_plan import bits_for_moduli, crt_constants, green_factor_packed, moduli_needed
from .tables import Fp64Recompute, IonDevice, tile_tasks
from .yk import yk_partial_matrices

__all__ = ["SplitEngine", "IonRows", "factors_for_grid", "host_tables", "choose_width", "DEFAULT_BITS"]

#: the split is at least this wide by default; ``bits=None`` then widens it to
#: what the same number of CRT moduli still holds exactly (free accuracy)
DEFAULT_BITS = 36


#: longest contraction the CRT kernel takes: its int32 accumulators are made
#: nonnegative by a bias of m * 2^18 >= kdim * 128^2 for every modulus m >= 223
KDIM_MAX = 3456


#: the single-ion contraction takes each table's tiles in blocks of
#: TASK_BLOCK x TASK_BLOCK (tables.tile_tasks): the tiles in flight then share
#: their residue panels in L2.  On the Z=70 table 8 measured fastest (2.87
#: against 2.92 ms row-major; 12 and 16 slower), with identical tables.
TASK_BLOCK = 8

#: doubles per row of the row record (screen bounds, |[X|Z]|, R_aa)
CB_STRIDE = 8
#: certificate limit: a table whose estimated Schwarz-relative split error
#: exceeds this is recomputed in FP64.  The estimate tracks the measured error
#: within a factor 0.7..3, so 2.5e-11 keeps every table below 1e-10.
CERT_LIMIT = 2.5e-11


def certify(grp_row0, grp_n, rowscale, cbound, limit: float, est, status, stream=None) -> None:
    """Enqueue the per-table certificate: est[g] and status[1] = count over limit."""
    L = _native.load()
    _native.check(L.rkb_split_certify(grp_row0.data_ptr(), grp_n.data_ptr(), grp_n.numel(), rowscale.data_ptr(),
                                      cbound.data_ptr(), float(limit), est.data_ptr(), status.data_ptr() + 4,
                                      _native.stream_handle(stream)), "rkb_split_certify")


def read_status(status, stream):
    """Copy the device status words to pinned host memory on the stream the
    work was enqueued on (None: the current stream) and wait for that stream
    (one synchronisation; the wait releases the GIL, unlike ``.item()``).
    Returns (stream, [words])."""
    s = stream if stream is not None else torch.cuda.current_stream()
    host = torch.empty(status.shape, dtype=status.dtype, pin_memory=True)
    with torch.cuda.stream(s):
        host.copy_(status, non_blocking=True)
    s.synchronize()
    return s, host.tolist()


def join_stream(s) -> None:
    """Make the current stream wait for work enqueued on ``s``."""
    cur = torch.cuda.current_stream()
    if s != cur:
        cur.wait_stream(s)


def check_kdim(kdim: int) -> None:
    if kdim > KDIM_MAX:
        raise ValueError(f"grid too long for the split engine: contraction length {kdim} > {KDIM_MAX} "
                         "(use precision='fp64')")


def choose_width(bits, n_mod, kdim: int) -> tuple[int, int]:
    """(bits, n_mod) for a contraction length: explicit values are kept;
    bits=None takes the widest split the moduli hold, and n_mod=None the
    fewest moduli for ``bits`` (DEFAULT_BITS when bits is None too).  Raises
    when the moduli cannot hold the products of the split exactly."""
    if n_mod is None:
        n_mod = moduli_needed(DEFAULT_BITS if bits is None else int(bits), kdim)
    n_mod = int(n_mod)
    held = bits_for_moduli(n_mod, kdim)
    bits = held if bits is None else int(bits)
    if bits > held:
        raise ValueError(f"{n_mod} moduli hold {held}-bit splits of length {kdim}, not {bits}")
    return bits, n_mod


_factor_cache: dict = {}
_factor_lock = threading.Lock()


def factors_for_grid(r_flat: np.ndarray, ng: int, ks, tau: float = 1e-3) -> dict:
    """k -> packed factor table for a grid (native factorisation, cached by
    grid content, k and tau)."""
    r_flat = np.ascontiguousarray(r_flat, dtype=np.float64)
    key0 = (hashlib.blake2b(r_flat.tobytes(), digest_size=16).hexdigest(), ng, tau)
    out = {}
    for k in ks:
        key = key0 + (int(k),)
        with _factor_lock:
            F = _factor_cache.get(key)
        if F is None:
            F = green_factor_packed(r_flat, ng, int(k), tau=tau)
            with _factor_lock:
                if len(_factor_cache) > 4096:
                    _factor_cache.clear()
                _factor_cache[key] = F
        out[int(k)] = F
    return out


_host_cache: dict = {}
#: host threads one host_tables call factorises its multipoles on (one: the
#: work is about 0.1 ms per multipole, and a serving planner pool already
#: runs requests side by side)
HOST_TABLE_THREADS = 1


def host_tables(r_flat: np.ndarray, ng: int, ks, tau: float = 1e-3) -> dict:
    """Host-side tables of a grid and multipole set, cached: the packed factor
    tables concatenated (``flat``, ``koff``), their Z counts, and the
    cell-minor copy the cell row kernel reads (``flat_t``, ``koff_t``).
    Pure host work, so a serving planner can prepare it off the launch path."""
    r_flat = np.ascontiguousarray(r_flat, dtype=np.float64)
    ks = tuple(int(k) for k in ks)
    key = (hashlib.blake2b(r_flat.tobytes(), digest_size=16).hexdigest(), ng, tau, ks)
    with _factor_lock:
        hit = _host_cache.get(key)
    if hit is not None:
        return hit
    nv = r_flat.shape[0] // ng
    n = nv * ng
    kmax = max(ks)
    mo, mi = yk_partial_matrices(ng)
    mo = np.ascontiguousarray(mo, dtype=np.float64)
    mi = np.ascontiguousarray(mi, dtype=np.float64)
    kk = np.asarray(ks, dtype=np.int32)
    cap1 = n + nv * ng * ng + n + ng + ng * ng + 2 + n * (ng + 1)
    flat = np.empty(len(ks) * cap1, dtype=np.float64)
    flat_t = np.empty(len(ks) * (2 * n + nv * ng * ng), dtype=np.float64)
    koff = np.empty(kmax + 1, dtype=np.int64)
    koff_t = np.empty(kmax + 1, dtype=np.int64)
    nz = np.empty(len(ks), dtype=np.int64)
    L = _native.load()
    # one native call (ctypes drops the interpreter lock for it): every
    # multipole factorised, the tables laid end to end, the cell-minor copy
    got = L.rkb_green_tables(r_flat.ctypes.data, nv, ng, kk.ctypes.data, len(ks), float(tau), mo.ctypes.data,
                             mi.ctypes.data, HOST_TABLE_THREADS, kmax, flat.ctypes.data, flat.shape[0],
                             koff.ctypes.data, flat_t.ctypes.data, flat_t.shape[0], koff_t.ctypes.data,
                             nz.ctypes.data)
    if got < 0:
        _native.check(int(-got), "rkb_green_tables")
    flat = flat[:got].copy()
    ends = [int(koff[k]) for k in ks[1:]] + [int(got)]
    factors = {k: flat[int(koff[k]):e] for k, e in zip(ks, ends)}
    out = {"factors": factors, "flat": flat, "koff": koff, "flat_t": flat_t, "koff_t": koff_t,
           "nz": {k: int(z) for k, z in zip(ks, nz)}}
    with _factor_lock:
        if len(_host_cache) > 256:
            _host_cache.clear()
        _host_cache[key] = out
    return out


CELLS_Z_MAX = 128  # Z columns per row of the cell-parallel row kernel
def _device_table(H: dict, key: str, device) -> torch.Tensor:
    """Device copy of one of a cached host-table set's arrays, kept with the set
    (the set is immutable and cached by grid content, so the copy is reused by
    every engine on that grid and device)."""
    cache = H.setdefault("_device", {})
    ck = (key, str(device))
    with _factor_lock:
        t = cache.get(ck)
    if t is None:
        t = torch.as_tensor(H[key], device=device)
        with _factor_lock:
            t = cache.setdefault(ck, t)
    return t


FUSED_PASSES_MAX = 32  # passes of 32 // ng cells kept in registers by the fused row kernel
FUSED_Z_MAX = 64


def fused_fits(nv: int, ng: int, max_z: int) -> bool:
    """Whether the register-resident row kernel takes this grid."""
    return 5 <= ng <= 11 and -(-(nv - 1) // (32 // ng)) <= FUSED_PASSES_MAX and max_z <= FUSED_Z_MAX


def cells_fit(nv: int, ng: int, max_z: int) -> bool:
    """Whether the cell-parallel row kernel takes this grid (one block of at
    most 256 threads: a thread per cell plus one per Z column)."""
    return 5 <= ng <= 11 and max_z <= CELLS_Z_MAX and -(-(nv + max_z) // 32) * 32 <= 256


def fused_body_width(nv: int, ng: int) -> int:
    """Residue positions spanned by the body in the fused layout (multiple of 128)."""
    passes = -(-(nv - 1) // (32 // ng))
    return 128 * (-(-passes // 4))


def fused_body_positions(nv: int, ng: int) -> np.ndarray:
    """Position of body column (m-1)*ng + node in the fused layout.

    The kernel takes cells from the last one down, 32 // ng cells per pass,
    lane = (cell offset within the pass) * ng + node; pass p of lane l is
    stored at 128*(p//4) + 4*l + p%4.
    """
    cpp = 32 // ng
    m = np.arange(1, nv)
    p, sub = np.divmod(nv - 1 - m, cpp)
    lane = sub[:, None] * ng + np.arange(ng)[None, :]
    pos = 128 * (p[:, None] // 4) + 4 * lane + (p[:, None] % 4)
    return pos.reshape(-1)


def _round_up(x: int, m: int) -> int:
    return (x + m - 1) // m * m


class IonRows:
    """Row side of the split engine for one ion: factor tables on the device,
    the residue layout (fused register kernel or two-kernel path) and the
    launch that writes the ion's rows into shared residue matrices."""

    KCHUNK = 128

    def __init__(self, dev: IonDevice, tau: float = 1e-3, fused: bool | None = None, rows_kernel: str | None = None,
                 device_tables: dict | None = None):
        """``device_tables``: the device copies of host_tables' flat, koff,
        flat_t, koff_t and the per-k Z counts (``zcount``), staged by the
        caller (tables.stage_ion); by default they are uploaded and cached
        with the grid's host tables."""
        self.dev = dev
        plan = dev.plan
        nv, ng = dev.nv, dev.ng
        r_host = dev.extra.get("r_host")
        if r_host is None:
            r_host = dev.r.detach().cpu().numpy()
        H = host_tables(r_host, ng, plan.ks, tau=tau)
        self.factors = H["factors"]
        kmax = max(plan.ks)
        d = dev.Pv.device
        dt = device_tables
        self.ktab = dt["flat"] if dt else _device_table(H, "flat", d)
        self.koff = dt["koff"] if dt else _device_table(H, "koff", d)
        self.kbody = (nv - 1) * ng
        self.nz = dict(H["nz"])
        max_z = max(self.nz.values())
        fits = fused_fits(nv, ng, max_z)
        if fused and not fits:
            raise ValueError(f"the fused row kernel does not fit this grid (nv={nv}, ng={ng}, Z columns {max_z})")

        # Three row kernels write the same residues:
        # * "cells": one block per row, one thread per cell (natural column
        #   order); the default wherever it fits;
        # * "fused": one warp per row in registers (permuted columns);
        # * "two": rows to an FP64 workspace, then residues (natural order).
        def gemm_work(body):
            return sum(plan.n_of_k(k) ** 2 * _round_up(body + self.nz[k], self.KCHUNK) for k in plan.ks)

        if fused is not None:
            kind = "fused" if fused else "two"
        elif rows_kernel is not None:
            kind = rows_kernel
        elif cells_fit(nv, ng, max_z):
            kind = "cells"
        elif fits and gemm_work(fused_body_width(nv, ng)) <= 1.05 * gemm_work(self.kbody):
            kind = "fused"
        else:
            kind = "two"
        if kind not in ("cells", "fused", "two"):
            raise ValueError(f"unknown row kernel {kind!r}")
        if kind == "cells" and not cells_fit(nv, ng, max_z):
            raise ValueError(f"the cell row kernel does not fit this grid (nv={nv}, ng={ng}, Z columns {max_z})")
        if kind == "fused" and not fits:
            raise ValueError(f"the fused row kernel does not fit this grid (nv={nv}, ng={ng}, Z columns {max_z})")
        self.kind = kind
        self.fused = kind == "fused"
        self.ktab_t = self.koff_t = None
        if kind == "cells":  # cell-minor copy of u, ell, C and L for coalesced per-cell reads
            self.ktab_t = dt["flat_t"] if dt else _device_table(H, "flat_t", d)
            self.koff_t = dt["koff_t"] if dt else _device_table(H, "koff_t", d)
        self.max_z = max_z
        self.body_w = fused_body_width(nv, ng) if self.fused else self.kbody
        self.kdim = {k: _round_up(self.body_w + self.nz[k], self.KCHUNK) for k in plan.ks}
        self.kmax_dim = max(self.kdim.values())
        self.has_z = max_z > 0
        if dt:
            self.zcount = dt["zcount"]
        else:
            zc = np.zeros(kmax + 1, dtype=np.int32)
            for k in plan.ks:
                zc[k] = self.nz[k]
            self.zcount = torch.as_tensor(zc, device=d)

    def column_positions(self, k: int) -> np.ndarray:
        """Residue position of every column of the row [X | Z] of multipole k."""
        nv, ng = self.dev.nv, self.dev.ng
        if not self.fused:
            return np.arange(self.kbody + self.nz[k])
        return np.concatenate([fused_body_positions(nv, ng), self.body_w + np.arange(self.nz[k])])

    def launch(self, bits: int, n_mod: int, moduli_c, resA, resB, kpad: int, row_base: int, nrows_total: int,
               rowscale, left, right, cbound, cwp: int, xwork, stream) -> None:
        """Write this ion's rows at rows [row_base, row_base + n_rows) of the
        [modulus][row][kpad] residue matrices (resA/resB, nrows_total rows)."""
        L = _native.load()
        dev, plan = self.dev, self.dev.plan
        rb = int(row_base)
        # the row range is folded into the base pointers (every modulus slab
        # shifts by the same row offset), so each launch sees rows from 0
        a_ptr = resA.data_ptr() + rb * kpad
        b_ptr = resB.data_ptr() + rb * kpad if resB is not None else 0
        rs, lf = rowscale.data_ptr() + 8 * rb, left.data_ptr() + 8 * rb * cwp
        rt, cb = right.data_ptr() + 8 * rb * cwp, cbound.data_ptr() + 8 * CB_STRIDE * rb
        if self.kind == "cells":
            _native.check(L.rkb_split_rows_cells(dev.Pv.data_ptr(), dev.Qv.data_ptr(), dev.n, dev.pairs.data_ptr(),
                                                 dev.row_pair.data_ptr(), dev.row_k.data_ptr(), plan.n_rows,
                                                 dev.w.data_ptr(), dev.nv, dev.ng, self.ktab.data_ptr(),
                                                 self.koff.data_ptr(), self.ktab_t.data_ptr(), self.koff_t.data_ptr(),
                                                 self.max_z, bits, n_mod, moduli_c, a_ptr,
                                                 b_ptr, kpad, 0, nrows_total, rs, lf, rt, cb, cwp,
                                                 _native.stream_handle(stream)),
                          "rkb_split_rows_cells")
            return
        if self.fused:
            _native.check(L.rkb_split_rows_fused(dev.Pv.data_ptr(), dev.Qv.data_ptr(), dev.n, dev.pairs.data_ptr(),
                                                 dev.row_pair.data_ptr(), dev.row_k.data_ptr(), plan.n_rows,
                                                 dev.w.data_ptr(), dev.nv, dev.ng, self.ktab.data_ptr(),
                                                 self.koff.data_ptr(), self.max_z, bits, n_mod, moduli_c, a_ptr,
                                                 b_ptr, kpad, 0, nrows_total, rs, lf, rt, cb, cwp,
                                                 _native.stream_handle(stream)),
                          "rkb_split_rows_fused")
            return
        _native.check(L.rkb_split_rows(dev.Pv.data_ptr(), dev.Qv.data_ptr(), dev.n, dev.pairs.data_ptr(),
                                       dev.row_pair.data_ptr(), dev.row_k.data_ptr(), plan.n_rows,
                                       dev.w.data_ptr(), dev.nv, dev.ng, self.ktab.data_ptr(), self.koff.data_ptr(),
                                       bits, n_mod, moduli_c, a_ptr, b_ptr, kpad, 0, nrows_total, rs, lf, rt, cb,
                                       cwp, xwork.data_ptr(), self.zcount.data_ptr(), _native.stream_handle(stream)),
                      "rkb_split_rows")


class SplitEngine:
    """Device buffers and launch plan of the split engine for one ion."""

    KCHUNK = 128

    def __init__(self, dev: IonDevice, bits: int | None = None, tau: float = 1e-3, n_mod: int | None = None,
                 corr_floor: float | None = None, fused: bool | None = None, materialize: bool = True,
                 rows_kernel: str | None = None, cert_limit: float = CERT_LIMIT):
        _native.require_device()
        self.dev = dev
        plan = dev.plan
        nv, ng = dev.nv, dev.ng
        self.ion_rows = R = IonRows(dev, tau=tau, fused=fused, rows_kernel=rows_kernel)
        self.factors, self.ktab, self.koff, self.kbody, self.nz = R.factors, R.ktab, R.koff, R.kbody, R.nz
        self.fused, self.max_z, self.body_w, self.kdim, self.zcount = R.fused, R.max_z, R.body_w, R.kdim, R.zcount
        d = dev.Pv.device
        self.kpad = max(self.kdim.values())
        check_kdim(self.kpad)
        self.bits, self.n_mod = choose_width(bits, n_mod, self.kpad)
        self.moduli, self.f_hi, self.f_lo, self.M, self.pair_inv = crt_constants(self.n_mod)
        self.cw = ng + 2  # g_0 and the two core-body coupling moments
        self.cwp = _round_up(self.cw, 2)
        nrows = plan.n_rows
        # rows padded to whole 128-row TMA boxes (zero rows never reach a stored entry)
        self.rows_alloc = _round_up(max(nrows, 1), 128)
        self.resA = torch.zeros((self.n_mod, self.rows_alloc, self.kpad), dtype=torch.int8, device=d)
        self.has_z = any(self.nz[k] > 0 for k in plan.ks)
        self.resB = torch.zeros_like(self.resA) if self.has_z else None
        self.rowscale = torch.empty(nrows, dtype=torch.float64, device=d)
        self.left = torch.empty((nrows, self.cwp), dtype=torch.float64, device=d)
        self.right = torch.empty_like(self.left)
        self.cbound = torch.empty((nrows, CB_STRIDE), dtype=torch.float64, device=d)
        # scratch of the two-kernel path: the FP64 rows [X | Z] before rounding
        self.xwork = (torch.empty((nrows, self.kpad), dtype=torch.float64, device=d) if R.kind == "two" else None)
        #: skip the FP64 core correction of a block when its bound is below
        #: 2^-(bits+10) of the block's scale (none of the entries can move by
        #: more than that; the split's own error is ~2^-bits of the same scale)
        self.corr_floor = 2.0 ** -(self.bits + 10) if corr_floor is None else float(corr_floor)
        sizes = [plan.n_of_k(k) for k in plan.ks]
        self.grp_row0 = torch.as_tensor([plan.k_row_offset[k] for k in plan.ks], dtype=torch.int64, device=d)
        self.grp_n = torch.as_tensor(sizes, dtype=torch.int64, device=d)
        self.grp_kdim = torch.as_tensor([self.kdim[k] for k in plan.ks], dtype=torch.int64, device=d)
        offs_out = np.concatenate([[0], np.cumsum(np.asarray(sizes, dtype=np.int64) ** 2)])
        self.grp_out = torch.as_tensor(offs_out[:-1], dtype=torch.int64, device=d)
        self.offsets = {k: int(offs_out[i]) for i, k in enumerate(plan.ks)}
        self.total = int(offs_out[-1])
        tasks = tile_tasks(sizes, block=TASK_BLOCK)
        self.n_tasks = int(tasks.shape[0])
        self.tasks = torch.as_tensor(tasks.reshape(-1), device=d)
        # task range of each group (tasks are grouped by multipole) for streaming
        bounds = np.searchsorted(tasks[:, 0], np.arange(len(sizes) + 1))
        self.task_range = [(int(bounds[i]), int(bounds[i + 1])) for i in range(len(sizes))]
        self.grp_out_zero = torch.zeros(len(sizes), dtype=torch.int64, device=d)
        #: [contraction status, number of tables whose certificate failed]
        self.status = torch.zeros(2, dtype=torch.int32, device=d)
        #: certificate estimate of every multipole table (Schwarz-relative error)
        self.est = torch.zeros(len(sizes), dtype=torch.float64, device=d)
        self.cert_limit = float(cert_limit)
        #: multipoles recomputed in FP64 by the last check_status()
        self.escalated: list = []
        self._stream = None
        #: the whole table (None when the engine only streams multipole tables)
        self.out = torch.empty(self.total, dtype=torch.float64, device=d) if materialize else None
        self._mod_c = (np.ctypeslib.as_ctypes(np.ascontiguousarray(self.moduli, dtype=np.int32)),
                       np.ctypeslib.as_ctypes(np.ascontiguousarray(self.f_hi)),
                       np.ctypeslib.as_ctypes(np.ascontiguousarray(self.f_lo)),
                       np.ctypeslib.as_ctypes(np.ascontiguousarray(np.concatenate([self.pair_inv, [1]]).astype(np.int32))))

    dominant_kernel = "split::crt_syrk_kernel"

    @property
    def launches_per_step(self) -> int:
        """Kernels per table run: the row kernel(s), the certificate, the contraction."""
        return 4 if self.ion_rows.kind == "two" else 3

    def column_positions(self, k: int) -> np.ndarray:
        """Residue position of every column of the row [X | Z] of multipole k."""
        return self.ion_rows.column_positions(k)

    #: when a list, rows() appends a (start, end) CUDA event pair around the
    #: row kernels, recorded on the launch stream
    row_events = None

    def rows(self, stream=None) -> None:
        """Row kernels, then the certificate of every table (both async)."""
        self._stream = stream
        ev = None
        if self.row_events is not None:
            s = stream if stream is not None else torch.cuda.current_stream()
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record(s)
        self.ion_rows.launch(self.bits, self.n_mod, self._mod_c[0], self.resA, self.resB, self.kpad, 0,
                             self.rows_alloc, self.rowscale, self.left, self.right, self.cbound, self.cwp,
                             self.xwork, stream)
        if ev is not None:
            ev[1].record(s)
            self.row_events.append(ev)
        certify(self.grp_row0, self.grp_n, self.rowscale, self.cbound, self.cert_limit, self.est, self.status,
                stream)

    #: when a list, contract() appends a (start, end) CUDA event pair around
    #: each contraction launch, recorded on the launch stream (live timing of
    #: the dominant kernel inside a caller's timed region)
    kernel_events = None

    def contract(self, stream=None) -> None:
        if self.out is None:
            raise ValueError("this engine streams its tables (materialize=False); use stream_tables()")
        if self.kernel_events is None:
            self._contract(self.grp_out, 0, self.n_tasks, self.out, stream)
            return
        s = stream if stream is not None else torch.cuda.current_stream()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        self._contract(self.grp_out, 0, self.n_tasks, self.out, s)
        b.record(s)
        self.kernel_events.append((a, b))

    def _contract(self, grp_out, t0, t1, out, stream) -> None:
        L = _native.load()
        _native.check(L.rkb_split_contract(self.resA.data_ptr(), _native.ptr(self.resB), self.kpad, self.rows_alloc,
                                           self.n_mod, self._mod_c[0], self._mod_c[3], self._mod_c[1], self._mod_c[2],
                                           self.M,
                                           self.rowscale.data_ptr(), self.left.data_ptr(), self.right.data_ptr(),
                                           self.cbound.data_ptr(), self.corr_floor, self.cw, self.cwp,
                                           self.grp_row0.data_ptr(), self.grp_n.data_ptr(),
                                           self.grp_kdim.data_ptr(), grp_out.data_ptr(),
                                           self.tasks.data_ptr() + 12 * t0, t1 - t0, out.data_ptr(),
                                           self.status.data_ptr(), _native.stream_handle(stream)),
                      "rkb_split_contract")

    def stream_tables(self, sink, stream=None, check: bool = True) -> None:
        """Compute the rows once, then each multipole's table into one of two
        rotating device buffers and hand it to ``sink(k, table, blocks, stream)``
        (see ``tables.stream_tables``); the whole table is never held.  The
        call waits once, after the row kernels, for the per-table certificate
        (tables that fail it are recomputed in FP64 before they reach the
        sink).  A sink with ``replaces_tables = True`` (one table per
        multipole, a later delivery of the same k replacing the earlier) is
        served without that wait: every table is contracted at once and
        ``check_status()`` recomputes a table whose certificate failed in FP64
        and delivers it again.  With ``check=False`` nothing else waits for the
        device: call ``check_status()`` once the stream's work is known to be
        done, to raise a contraction error."""
        s = stream if stream is not None else torch.cuda.current_stream()
        plan = self.dev.plan
        self.rows(s)
        self._sink = sink
        if getattr(sink, "replaces_tables", False):
            # the sink keeps one table per multipole and takes a later
            # delivery of the same k in its place: every table is contracted
            # at once, without waiting for the certificate, and check_status()
            # recomputes a failing table in FP64 and delivers it again
            fp64 = set()
            self._deferred = True
        else:
            # which tables go to FP64 is known from the rows alone: one wait
            # here, on this stream only and without holding the GIL (serving
            # launches requests from several host threads)
            _, (_, flagged) = read_status(self.status, s)
            fp64 = set(self._failing(self.est.cpu().numpy())) if flagged else set()
            self._deferred = False
        self.escalated = sorted(fp64)
        nmax = max(plan.n_of_k(k) for k in plan.ks)
        bufs = [torch.empty(nmax * nmax, dtype=torch.float64, device=self.resA.device) for _ in range(2)]
        #: device bytes the engine holds while streaming (buffers included)
        self.held_bytes = self.device_bytes() + sum(b.numel() * 8 for b in bufs)
        for gi, k in enumerate(plan.ks):
            nk = plan.n_of_k(k)
            t0, t1 = self.task_range[gi]
            buf = bufs[gi % 2][:nk * nk]
            if k in fp64:
                self._recompute(((k, 0),)).run(buf, s)
            elif self.kernel_events is not None:
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(s)
                self._contract(self.grp_out_zero, t0, t1, buf, s)
                b.record(s)
                self.kernel_events.append((a, b, k))
            else:
                self._contract(self.grp_out_zero, t0, t1, buf, s)
            sink(k, buf.view(nk, nk), plan.block_ranges_of_k(k), s)
        self._bufs = bufs  # kept alive until the caller has waited for the stream
        self._streamed = True
        if check:
            self.check_status()

    def run_to_host(self, host: torch.Tensor, stream=None, copy_stream=None, packed: bool = False) -> None:
        """The whole table into ``host`` (pinned, ``total`` doubles): the rows
        and the certificate, then each multipole's table is contracted (or
        recomputed in FP64 when its certificate failed) on ``stream`` and copied
        to the host on ``copy_stream`` while the next one is contracted.
        ``packed``: each table's upper triangle only, at the packed offsets
        of tables.packed_offsets (unique_entries doubles in all).
        Returns once the host copy is complete; raises like check_status()."""
        if self.out is None:
            raise ValueError("this engine streams its tables (materialize=False); use stream_tables()")
        need = self.dev.plan.unique_entries if packed else self.total
        if host.numel() < need or host.is_cuda:
            raise ValueError(f"host buffer must be a CPU tensor of at least {need} doubles")
        s = stream if stream is not None else torch.cuda.current_stream()
        cs = copy_stream if copy_stream is not None else self.__dict__.setdefault(
            "_copy_stream", torch.cuda.Stream(device=self.out.device))
        plan = self.dev.plan
        self.rows(s)
        _, (_, flagged) = read_status(self.status, s)  # which tables go to FP64: one wait
        fp64 = set(self._failing(self.est.cpu().numpy())) if flagged else set()
        self.escalated = sorted(fp64)
        from .tables import PackedShipper
        shipper = PackedShipper(plan, host, self.out.device, cs) if packed else None
        for gi, k in enumerate(plan.ks):
            nk, o = plan.n_of_k(k), self.offsets[k]
            if k in fp64:
                self._recompute(((k, o),)).run(self.out, s)
            else:
                t0, t1 = self.task_range[gi]
                self._contract(self.grp_out, t0, t1, self.out, s)
            if shipper is not None:
                shipper.ship(k, self.out.data_ptr() + 8 * o, s)
                continue
            ev = torch.cuda.Event()
            ev.record(s)
            cs.wait_event(ev)
            with torch.cuda.stream(cs):
                host[o:o + nk * nk].copy_(self.out[o:o + nk * nk], non_blocking=True)
        self._streamed = True  # the per-table route is already taken
        try:
            self.check_status()
        finally:
            cs.synchronize()

    def run(self, stream=None, upload: bool = True, check: bool = True) -> torch.Tensor:
        self.rows(stream)
        self.contract(stream)
        if check:
            self.check_status()
        return self.out

    def device_bytes(self) -> int:
        """Bytes of the engine's own device buffers (not the ion's inputs)."""
        ts = [self.ktab, self.koff, self.resA, self.resB, self.rowscale, self.left, self.right, self.cbound,
              self.xwork, self.zcount, self.tasks, self.est, self.out]
        return int(sum(t.numel() * t.element_size() for t in ts if t is not None))

    def _failing(self, est) -> list:
        return [k for gi, k in enumerate(self.dev.plan.ks) if not est[gi] <= self.cert_limit]

    def check_status(self) -> None:
        """Wait for the device, raise a contraction error, and recompute in FP64
        (on the launch stream) every table whose certificate failed; the
        multipoles recomputed are listed in ``escalated``."""
        s, (st, flagged) = read_status(self.status, self._stream)
        if st:
            self.status[0] = 0
            _native.check(st, "crt_syrk_kernel")
        if getattr(self, "_streamed", False):  # the stream path chose per table already
            self._streamed = False
            if getattr(self, "_deferred", False):
                self._deferred = False
                self.escalated = self._failing(self.est.cpu().numpy()) if flagged else []
                plan = self.dev.plan
                for k in self.escalated:  # recompute in FP64 and deliver again
                    nk = plan.n_of_k(k)
                    buf = torch.empty(nk * nk, dtype=torch.float64, device=self.resA.device)
                    self._recompute(((k, 0),)).run(buf, s)
                    self._sink(k, buf.view(nk, nk), plan.block_ranges_of_k(k), s)
                if self.escalated:
                    s.synchronize()
            return
        self.escalated = []
        if flagged and self.out is not None:
            self.escalated = self._failing(self.est.cpu().numpy())
            self._recompute(tuple((k, self.offsets[k]) for k in self.escalated)).run(self.out, s)
            join_stream(s)

    def _recompute(self, key) -> Fp64Recompute:
        """FP64 recomputation plan for (k, output offset) groups, cached."""
        cache = self.__dict__.setdefault("_recompute_cache", {})
        plan = cache.get(key)
        if plan is None:
            plan = cache[key] = Fp64Recompute([(self.dev, k, o) for k, o in key])
        return plan

    def info(self) -> dict:
        return {"bits": self.bits, "n_mod": self.n_mod, "moduli": [int(m) for m in self.moduli], "fused": self.fused,
                "rows_kernel": self.ion_rows.kind, "cert_limit": self.cert_limit,
                "fp64_multipoles": list(self.escalated),
                "kpad": self.kpad, "z_columns": {int(k): v for k, v in self.nz.items()},
                "device_bytes": self.device_bytes(),
                "tasks": self.n_tasks}

    def int8_ops(self, ks=None) -> tuple[float, float]:
        """(algorithmic, issued) int8 tensor ops of the contraction of the
        multipoles ``ks`` (all by default): 2 * kdim ops per modulus for every
        unique entry (i <= j) of every table; the tiles actually issued also
        cover the lower half of diagonal tiles and the padding of edge tiles."""
        plan = self.dev.plan
        ops, issued = 0.0, 0.0
        for k in (plan.ks if ks is None else ks):
            nk = plan.n_of_k(k)
            nt = (nk + 127) // 128
            ops += 2.0 * self.n_mod * self.kdim[k] * (nk * (nk + 1) // 2)
            issued += 2.0 * self.n_mod * self.kdim[k] * (nt * (nt + 1) // 2) * 128 * 128
        return ops, issued

    def row_bytes(self) -> int:
        """Algorithmic HBM bytes of the row kernels: the orbital values read
        once, the int8 residue matrices (and their Z-negated copy) and the
        per-row scale, core vectors and row records written."""
        d = self.dev
        reads = (d.Pv.numel() + d.Qv.numel()) * 8
        res = self.n_mod * self.dev.plan.n_rows * self.kpad * (2 if self.resB is not None else 1)
        per_row = 8 + 2 * 8 * self.cwp + 8 * 8
        return int(reads + res + self.dev.plan.n_rows * per_row)

    def roofline(self, stream=None, flush=None, reps: int = 3, kernel_ms: float | None = None) -> dict:
        """Roofline of the dominant kernel (K3s): its duration ``kernel_ms``
        (e.g. the mean of the launches recorded through ``kernel_events``
        inside a timed region), or else timed alone with CUDA events on
        ``stream`` over ``reps`` launches."""
        import json
        import os
        if kernel_ms is None:
            s = stream or torch.cuda.current_stream()
            self.rows(s)
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
            for a, b in ev:
                if flush is not None:
                    flush.zero_()
                a.record(s)
                self.contract(s)
                b.record(s)
            torch.cuda.synchronize()
            self.check_status()
            ms = float(np.median([a.elapsed_time(b) for a, b in ev]))
        else:
            ms = float(kernel_ms)
        plan = self.dev.plan
        ops, issued = self.int8_ops()
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        peaks_path = os.path.join(root, "MEASURED_PEAKS.json")
        if os.path.exists(peaks_path):
            with open(peaks_path) as f:
                bf16 = float(json.load(f)["bf16_tflops"])
            src = "MEASURED_PEAKS.json bf16_tflops x 2 (dense int8 issues at twice the bf16 rate on B200)"
        else:
            bf16, src = 1590.0, "fallback 1.59 PFLOP/s bf16 x 2"
        peak = 2.0 * bf16
        ach = ops / (ms / 1e3) / 1e12
        return {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TOP/s (int8)", "frac": ach / peak,
                "traffic": None, "kernel": self.dominant_kernel, "kernel_ms": ms, "peak_source": src,
                "algorithmic_int8_ops": ops, "issued_int8_ops": issued, "unit_of_work": "unique entry",
                "units_per_launch": int(plan.unique_entries), "n_mod": self.n_mod, "bits": self.bits}
