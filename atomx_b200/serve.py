"""Serving loop for Slater-table requests on one GPU (continuous batching).

A request carries one ion: its radial basis, its spinor coefficients and
kappas, and k_max. This is what an SCF or CI client holds when it asks for
R^k tables. The server runs each request through three stages:

1. planning, in a worker pool: the pair/row plan and, for the split engine,
   the factored Green operators of the grid and their packed host tables
   (one native call, cached by grid content); then the request's device
   inputs, staged on the planners' staging stream (coefficients, orbital
   values, basis and plan arrays, the split engine's factor tables);
2. admission in groups: when a stream slot is free, the requests at the head
   of the ready queue (arrival order) form the next group while it holds at
   most ``max_group`` requests and at most ``group_bytes`` of device memory,
   and it fits the HBM budget beside the groups already on the GPU. The
   footprint of a group is every request's coefficients, orbital values and
   whole tables, and every ion's residue or (g, Y) rows at the group's
   largest row width;
3. device work, on the slot's CUDA stream and set up by the slot's launcher
   thread: every ion's row kernels (spread over the slot's side streams) and
   ONE contraction launch over the tiles of every (ion, k) table of the group
   (``batch.SplitBatch`` / ``batch.Fp64Batch``, their buffers carved from the
   slot's reusable ``batch.Workspace``). Each table then goes to its
   request's sink with its kappa-block ranges. The launcher waits (without
   the GIL) for an event after the last table, completes the group (for
   sinks that take a table again, tables whose split certificate failed are
   recomputed in FP64 and delivered again) and frees the slot.

A request too large to hold whole (above ``group_bytes`` on its own) runs
alone on the streaming engine instead: one multipole table at a time through
two rotating buffers (``tables.stream_tables``).

Under light load a group is one request and the loop is a queue with
overlapping slots; when requests arrive faster than the device retires them,
the queue grows while both slots are busy and the next group takes all of
it, so the host set-up and the device's small launches are shared by the
group and throughput rises with the load.

Latency is completion minus arrival on the server clock. ``serve`` returns
p50/p99 latency, throughput (ordered R^k entries per second), the group
sizes and the tables recomputed in FP64. Each result is independent of the
mix it ran in: every split request uses the same CRT moduli (SERVE_N_MOD)
and correction floor (SERVE_CORR_FLOOR), its split width follows from its
own contraction length, and the kernels are deterministic and take no input
from other ions, so a request gives the same tables alone and in any group;
``tests/test_gpu_serve.py`` checks that.
"""
from __future__ import annotations

import gc
import threading
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np
import torch

from .batch import Fp64Batch, SplitBatch, Workspace
from .device import wait_for
from .plan import make_plan
from .split import KDIM_MAX, IonRows, check_kdim, host_tables
from .split_plan import bits_for_moduli, moduli_needed
from .tables import evaluate_staged, stage_ion, upload_ion

__all__ = ["Request", "ServeReport", "SlaterServer", "ChecksumSink", "footprint_bytes", "footprint_parts",
           "P99_BOUND_MS", "SERVE_N_MOD", "SERVE_CORR_FLOOR", "GROUP_BYTES"]

#: The latency bound the loop is held to on the mixed-ion stream (Poisson
#: arrivals at 200 requests/s, Z 2..92, 30..200 B-splines, 10..300 spinors,
#: k_max 2..14): the 99th percentile of (last table delivered - arrival),
#: with two stream slots.
P99_BOUND_MS = 500.0

#: CRT moduli of every served split request.  Eleven moduli hold a split of at
#: least 37 bits at every contraction length the split engine takes
#: (KDIM_MAX), and each request takes the widest split they hold at its own
#: contraction length, so a request's width depends on its grid alone.
SERVE_N_MOD = 11
#: FP64 core-correction floor of every served split request: 2^-(b + 10) for
#: the narrowest width b that SERVE_N_MOD moduli give (37 bits).
SERVE_CORR_FLOOR = 2.0 ** -(bits_for_moduli(SERVE_N_MOD, KDIM_MAX) + 10)
#: A group holds at most this many bytes of device memory (whole tables, rows
#: and inputs); a request that needs more alone runs on the streaming engine.
GROUP_BYTES = 24 << 30
#: side streams per slot for the row kernels of a group's ions
ROW_STREAMS = 4


@dataclass
class Request:
    """One Slater-table request (an ion with its orbitals) and its timings."""
    rid: int
    ion: object                    # workloads.Ion: basis, coefficients, kappas
    k_max: int
    arrival: float = 0.0           # seconds on the server clock
    sink: object = None            # sink(k, table, blocks, stream); default ChecksumSink
    plan: object = None
    footprint: int = 0
    planned: float | None = None
    admitted: float | None = None
    done: float | None = None
    entries: int = 0
    error: BaseException | None = None
    state: dict = field(default_factory=dict)
    timing: dict = field(default_factory=dict)   # host planning and launch times (ms)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


class ChecksumSink:
    """Consumes every table on the device: per-(k, kappa-block) sums.  It
    keeps one result per multipole, so a later delivery of the same k (a
    table recomputed after a failed certificate) replaces the earlier one."""

    replaces_tables = True

    def __init__(self):
        self.sums = {}

    def __call__(self, k, table, blocks, stream):
        with torch.cuda.stream(stream):
            self.sums[k] = table.sum(dim=1)  # one value per row, kept per k


@dataclass
class ServeReport:
    n: int
    wall_s: float
    entries: int
    latencies_ms: list
    queue_ms: list
    precision: str
    max_inflight_seen: int
    stages_ms: dict = field(default_factory=dict)   # stage -> per-request times (ms)
    group_sizes: list = field(default_factory=list)  # requests per admitted group
    fp64_tables: int = 0                              # split tables recomputed in FP64
    tail: list = field(default_factory=list)          # timelines of the slowest 1 % of requests

    def summary(self) -> dict:
        lat = np.asarray(self.latencies_ms)
        q = np.asarray(self.queue_ms)
        stages = {f"{k}_p50": float(np.percentile(v, 50)) for k, v in self.stages_ms.items() if v}
        return {"requests": self.n, "wall_s": self.wall_s, "entries": self.entries, "stages_ms": stages,
                "throughput_entries_per_s": self.entries / self.wall_s if self.wall_s > 0 else None,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "max_ms": float(lat.max()), "queue_p50_ms": float(np.percentile(q, 50)),
                "queue_p99_ms": float(np.percentile(q, 99)), "precision": self.precision,
                "max_inflight": self.max_inflight_seen, "groups": len(self.group_sizes),
                "group_size_mean": float(np.mean(self.group_sizes)) if self.group_sizes else 0.0,
                "group_size_max": int(max(self.group_sizes, default=0)), "fp64_tables": self.fp64_tables,
                "tail": self.tail}


def footprint_parts(ion, plan, precision: str, whole_tables: bool = False) -> tuple[int, int, int, int]:
    """A request's device bytes as (fixed, rows, width, bytes per row and
    column): the total is fixed + rows * width * bytes.  ``width`` is the row
    length the engine pads to (residue or FP64 row columns); in a group every
    ion's rows take the group's largest width.  With ``whole_tables`` every
    table is held at once (a request in a group), else the streaming engine's
    two rotating table buffers."""
    nv, ng = ion.bsp["gr"].shape
    n = nv * ng
    n_orb = ion.P.shape[0]
    rows = plan.n_rows
    if whole_tables:
        tabs = 8 * sum(plan.n_of_k(k) ** 2 for k in plan.ks)
    else:
        tabs = 2 * 8 * max(plan.n_of_k(k) for k in plan.ks) ** 2
    fixed = 8 * (2 * n_orb * n + ion.P.size + ion.Q.size) + tabs + 64 * rows
    if precision == "split":
        kpad = 128 * (-(-((nv - 1) * ng + 64) // 128))
        n_mod = max(SERVE_N_MOD, moduli_needed(36, kpad))
        # two int8 residue copies per modulus (128 rows of padding) and the
        # FP64 workspace of the two-kernel row path
        return fixed + 2 * n_mod * 128 * kpad + 8 * rows * 48, rows, kpad, 2 * n_mod + 8
    return fixed, rows, 32 * (-(-n // 32)), 2 * 8


def footprint_bytes(ion, plan, precision: str, whole_tables: bool = False) -> int:
    """Device bytes a request holds while it runs alone (an upper estimate)."""
    fixed, rows, width, per = footprint_parts(ion, plan, precision, whole_tables)
    return fixed + rows * width * per


def _group_footprint(reqs) -> int:
    """Device bytes of a group of planned requests: their fixed parts, and
    every ion's rows at the group's largest width."""
    parts = [r.state.get("parts") or (r.footprint, 0, 0, 0) for r in reqs]
    rows = sum(p[1] for p in parts)
    return sum(p[0] for p in parts) + rows * max(p[2] for p in parts) * max(p[3] for p in parts)


@dataclass
class _Slot:
    """A stream slot: the stream a group runs on, the side streams its row
    kernels spread over, and the device workspace its batches reuse (tables,
    residues and rows of one group at a time, so groups after the first few
    allocate no device memory)."""
    stream: object
    side: list
    ws: object


class SlaterServer:
    """Continuous-batching server for R^k table requests on the current GPU.

    ``max_inflight`` stream slots each run one group of requests at a time;
    a group holds up to ``max_group`` requests and at most ``group_bytes`` of
    device memory (whole tables, rows and inputs).  A request larger than
    that alone runs on the streaming engine."""

    def __init__(self, precision: str = "split", hbm_budget: int | None = None, max_inflight: int = 2,
                 workers: int = 4, bits: int | None = None, max_group: int = 16, group_bytes: int = GROUP_BYTES):
        if precision not in ("split", "fp64"):
            raise ValueError(f"unknown precision {precision!r}")
        self.precision, self.max_inflight, self.bits = precision, int(max_inflight), bits
        self.max_group, self.group_bytes = int(max_group), int(group_bytes)
        if self.max_inflight < 1 or self.max_group < 1:
            raise ValueError("max_inflight and max_group must be >= 1")
        # Blocks the caching allocator keeps for other streams (earlier work in
        # this process) are given back first: left cached, they can fill the
        # device under a request and force a flush (a device-wide
        # synchronisation) mid-stream, and they would shrink the budget.
        torch.cuda.empty_cache()
        if hbm_budget is None:
            free, total = torch.cuda.mem_get_info()
            hbm_budget = int(0.6 * free)
        self.hbm_budget = int(hbm_budget)
        self.device = torch.cuda.current_device()
        self.pool = ThreadPoolExecutor(max_workers=workers)
        # one launcher thread per stream slot: a group's set-up and launches
        # run there, and the thread then waits (without the GIL) for the
        # group's completion event, so the loop itself only admits and retires
        self.launchers = ThreadPoolExecutor(max_workers=self.max_inflight)
        self.slots = [_Slot(torch.cuda.Stream(), [torch.cuda.Stream() for _ in range(ROW_STREAMS)], Workspace())
                      for _ in range(self.max_inflight)]
        # each slot holds its share of the budget in one buffer from the start,
        # so no group allocates device memory
        reserve = min(self.group_bytes, self.hbm_budget // self.max_inflight)
        if reserve >= Workspace.MIN_CHUNK:
            for slot in self.slots:
                with torch.cuda.stream(slot.stream):
                    slot.ws.reserve(reserve)
        self._stage_stream, self._stage_lock = None, threading.Lock()
        self._tls = threading.local()  # per planner thread: its pinned staging buffer
        self._t0 = time.perf_counter()

    def _now(self) -> float:
        return time.perf_counter() - self._t0

    # ---------------------------------------------------------------- stages
    def _plan(self, req: Request) -> Request:
        t0 = time.perf_counter()
        req.plan = make_plan(req.ion.kappa, req.k_max)
        for k in req.plan.ks:  # the sinks' kappa-block ranges, built here rather than by the launcher
            req.plan.block_ranges_of_k(k)
        if self.precision == "split":
            host_tables(np.asarray(req.ion.bsp["gr"], dtype=np.float64).reshape(-1), req.ion.bsp["gr"].shape[1],
                        req.plan.ks)
        parts = footprint_parts(req.ion, req.plan, self.precision, whole_tables=True)
        req.state["streamed"] = parts[0] + parts[1] * parts[2] * parts[3] > self.group_bytes
        if req.state["streamed"]:
            parts = footprint_parts(req.ion, req.plan, self.precision)
        req.state["parts"] = parts
        req.footprint = parts[0] + parts[1] * parts[2] * parts[3]
        req.entries = req.plan.ordered_entries
        t1 = time.perf_counter()
        self._stage(req)
        req.timing["plan_ms"] = 1e3 * (t1 - t0)
        req.timing["stage_ms"] = 1e3 * (time.perf_counter() - t1)
        return req

    def _planner_stream(self):
        # one staging stream for every planner thread: the caching allocator
        # keeps freed blocks per stream, so staged inputs then share one pool
        if self._stage_stream is None:
            with self._stage_lock:
                if self._stage_stream is None:
                    with torch.cuda.device(self.device):
                        self._stage_stream = torch.cuda.Stream()
        return self._stage_stream

    def _stage(self, req: Request) -> None:
        """A request's device inputs, prepared by its planner thread on the
        staging stream, off the launch path (``tables.stage_ion``):
        coefficients, the basis and plan arrays and, for the split engine,
        the factor tables, in one device allocation and one copy from the
        thread's pinned buffer, and the split engine's row side.  The
        orbital values (K1) are evaluated later, on the group's stream: a
        kernel on the staging stream would wait for SMs behind a running
        contraction, and the planners with it.  A new radial grid would otherwise make these a
        dozen synchronous copies on the launch path.  They are small beside
        the tables (orbital values: 16 bytes per spinor and grid node)."""
        ps = self._planner_stream()
        split = self.precision == "split" and not req.state["streamed"]
        H = None
        if split:
            H = host_tables(np.asarray(req.ion.bsp["gr"], dtype=np.float64).reshape(-1),
                            req.ion.bsp["gr"].shape[1], req.plan.ks)
        with torch.cuda.device(self.device), torch.cuda.stream(ps):
            dev, dtab, pinned = stage_ion(req.ion, req.plan, ps, getattr(self._tls, "pinned", None), H,
                                          evaluate=False)
            rows = IonRows(dev, device_tables=dtab) if split else None
        self._tls.pinned = pinned
        wait_for(ps)  # the launcher's stream reads them; the pinned buffer is free again
        if rows is not None:
            check_kdim(rows.kmax_dim)  # a grid the split engine does not take fails this request alone
        req.state["dev"], req.state["ion_rows"] = dev, rows

    @staticmethod
    def _dev(req: Request, stream):
        dev = req.state.get("dev")
        if dev is None:
            return upload_ion(req.ion, k_max=req.k_max, plan=req.plan, stream=stream)
        evaluate_staged(dev, stream)  # K1 on the group's stream, ahead of its rows
        return dev

    def _batch(self, group: list, slot: _Slot):
        """One batch over the group's ions on the slot's stream; every table
        goes to its request's sink.  Returns the completion step (deferred
        certificates)."""
        s = slot.stream
        devs = [self._dev(r, s) for r in group]
        # the slot's previous group, and its sinks' work, completed before
        # this launcher returned: its workspace views are free again
        slot.ws.reset()
        split = self.precision == "split"
        if split:
            rows = [r.state.get("ion_rows") for r in group]
            b = SplitBatch(devs, bits=self.bits, n_mod=SERVE_N_MOD, ion_widths=True, corr_floor=SERVE_CORR_FLOOR,
                           ion_rows=rows if all(x is not None for x in rows) else None, workspace=slot.ws)
            b.step(s, slot.side)
        else:
            b = Fp64Batch(devs, workspace=slot.ws)
            b.step(s)
        deferred = split and all(getattr(r.sink, "replaces_tables", False) for r in group)
        if split and not deferred:
            # one wait (without the GIL): tables whose certificate failed are
            # recomputed in FP64 before any table reaches a sink
            b.check_status()
        for i, r in enumerate(group):
            for k in r.plan.ks:
                r.sink(k, b.table(i, k), r.plan.block_ranges_of_k(k), s)

        def complete():
            if deferred:
                b.check_status()  # the device is done: recompute failing tables in FP64 ...
                for i, k in b.escalated:  # ... and deliver them again
                    r = group[i]
                    r.sink(k, b.table(i, k), r.plan.block_ranges_of_k(k), s)
                if b.escalated:
                    wait_for(s)
            return len(b.escalated) if split else 0
        return complete

    def _stream_one(self, req: Request, slot: _Slot):
        """A request too large to hold whole: the streaming engine, one table
        at a time through two rotating buffers."""
        from . import tables as T
        s = slot.stream
        dev = self._dev(req, s)
        if self.precision == "split":
            from .split import SplitEngine
            eng = SplitEngine(dev, bits=self.bits, materialize=False)
            eng.stream_tables(req.sink, stream=s, check=False)

            def complete():
                eng.check_status()
                return len(eng.escalated)
            return complete
        T.stream_tables(dev, req.sink, precision="fp64", stream=s)
        return lambda: 0

    def _run_group(self, group: list, slot: _Slot) -> int:
        """Launcher thread: enqueue the group, wait for it, complete it.
        Returns the number of its tables recomputed in FP64."""
        t_launch = time.perf_counter()
        t_enq, fp64 = None, 0
        for r in group:
            if r.sink is None:
                r.sink = ChecksumSink()
        s = slot.stream
        try:
            with torch.cuda.device(self.device), torch.cuda.stream(s):
                if len(group) == 1 and group[0].state.get("streamed"):
                    complete = self._stream_one(group[0], slot)
                else:
                    complete = self._batch(group, slot)
                # the launcher sleeps until the group is done (a blocking-sync
                # event: no core spent spinning, see device.wait_for)
                ev = torch.cuda.Event(blocking=True)
                ev.record(s)
                t_enq = time.perf_counter()
                ev.synchronize()
                fp64 = complete()
        except BaseException as exc:  # a failed group does not stop the server
            for r in group:
                r.error = exc
            try:  # buffers return to the stream's pool: let enqueued work finish
                s.synchronize()
            except BaseException:
                pass
        t_done = time.perf_counter()
        done = self._now()
        for r in group:
            r.done = done
            r.timing["group"] = len(group)
            if t_enq is not None:
                r.timing["launch_host_ms"] = 1e3 * (t_enq - t_launch)
                r.timing["after_enqueue_ms"] = 1e3 * (t_done - t_enq)
        return fp64

    # ------------------------------------------------------------------ loop
    def _take_group(self, ready: deque, used: int, busy: bool) -> tuple[list, int]:
        """The next group and its device bytes, FIFO: requests join while the
        group holds at most max_group requests and group_bytes of device
        memory, and fits the HBM budget beside the groups in flight (the
        first request of an idle device always starts; a streamed request
        runs alone)."""
        group, fp = [], 0
        while ready and len(group) < self.max_group:
            r = ready[0]
            if group and (r.state.get("streamed") or group[0].state.get("streamed")):
                break
            nxt = _group_footprint(group + [r])
            if group and nxt > self.group_bytes:
                break
            if (busy or group) and used + nxt > self.hbm_budget:
                break
            group.append(ready.popleft())
            fp = nxt
        return group, fp

    def serve(self, requests: list[Request], realtime: bool = True, pause_gc: bool = True) -> ServeReport:
        """Run the requests (sorted by arrival) to completion; return timings.
        ``realtime``: requests arrive at their arrival times; otherwise all
        arrive at once and are planned before the first group starts.

        ``pause_gc``: collect once before the clock starts, then keep
        Python's cyclic garbage collector off while serving (its previous
        state is restored on return).  A full collection walks every object
        of the process while holding the GIL; in a process with a large heap
        that is a pause of a large fraction of a second in which no request
        is planned or launched.  Reference counting still frees the
        requests' objects as they complete."""
        was_enabled = gc.isenabled()
        if pause_gc:
            gc.collect()
            gc.disable()
        try:
            return self._serve(requests, realtime)
        finally:
            if pause_gc and was_enabled:
                gc.enable()

    def _serve(self, requests: list[Request], realtime: bool) -> ServeReport:
        todo = deque(sorted(requests, key=lambda r: r.arrival))
        planning, ready, inflight, free_slots = [], deque(), [], list(self.slots)
        used = 0
        max_seen = 0
        groups, fp64 = [], 0
        self._t0 = time.perf_counter()
        now = self._now
        # The loop sleeps until something changes: a plan or a group completes
        # (their futures set `wake`) or the next request arrives.  Waking at a
        # fixed short period instead would take the GIL thousands of times a
        # second from the planners and launchers.
        wake = threading.Event()

        def notify(_fut):
            wake.set()

        while todo or planning or ready or inflight:
            wake.clear()
            t = now()
            # arrivals: (in real time, or all at once when not realtime)
            while todo and (not realtime or todo[0].arrival <= t):
                r = todo.popleft()
                if not realtime:
                    r.arrival = t
                fut = self.pool.submit(self._plan, r)
                fut.add_done_callback(notify)
                planning.append((r, fut))
            # planned requests join the ready queue in arrival order
            still = []
            for r, fut in planning:
                if fut.done():
                    r.planned = now()
                    if fut.exception() is not None:  # e.g. an invalid request
                        r.error, r.done = fut.exception(), r.planned
                        r.state.clear()
                    else:
                        ready.append(r)
                else:
                    still.append((r, fut))
            planning = still
            if len(ready) > 1:
                ready = deque(sorted(ready, key=lambda r: r.arrival))
            # completions: the launcher thread has seen the group's event fire
            # and completed it
            for item in list(inflight):
                group, gfp, slot, fut = item
                if not fut.done():
                    continue
                if fut.exception() is None:
                    fp64 += fut.result()
                for r in group:
                    if r.error is None and fut.exception() is not None:
                        r.error = fut.exception()
                    if r.done is None:
                        r.done = now()
                    r.state.clear()
                used -= gfp
                free_slots.append(slot)
                inflight.remove(item)
            # admission: groups by slots and HBM footprint (all requests present
            # at once, when not realtime, are planned before the first group)
            admitted = False
            while ready and free_slots and (realtime or not planning):
                group, gfp = self._take_group(ready, used, bool(inflight))
                if not group:
                    break
                admitted = True
                slot = free_slots.pop()
                ta = now()
                for r in group:
                    r.admitted = ta
                used += gfp
                groups.append(len(group))
                fut = self.launchers.submit(self._run_group, group, slot)
                fut.add_done_callback(notify)
                inflight.append((group, gfp, slot, fut))
                max_seen = max(max_seen, sum(len(g[0]) for g in inflight))
            if not admitted:
                # until the next arrival at most (a future that completed
                # since the clear() above has set the event already)
                timeout = 0.05
                if realtime and todo:
                    timeout = min(timeout, max(0.0, todo[0].arrival - now()))
                wake.wait(timeout)
        wall = now()
        done = [r for r in requests if r.error is None]
        stages = {k: [r.timing[k] for r in done if k in r.timing]
                  for k in ("plan_ms", "stage_ms", "launch_host_ms", "after_enqueue_ms")}
        # where the slowest requests spent their time (server clock, ms)
        slow = sorted(done, key=lambda r: r.latency, reverse=True)[:max(3, len(done) // 100)]
        tail = [dict({"rid": r.rid, "arrival": 1e3 * r.arrival, "planned": 1e3 * (r.planned - r.arrival),
                      "admitted": 1e3 * (r.admitted - r.arrival), "done": 1e3 * r.latency, "entries": r.entries},
                     **{k: round(v, 2) for k, v in r.timing.items()}) for r in slow]
        return ServeReport(n=len(requests), wall_s=wall, entries=int(sum(r.entries for r in done)),
                           latencies_ms=[1e3 * r.latency for r in done],
                           queue_ms=[1e3 * (r.admitted - r.arrival) for r in done], precision=self.precision,
                           max_inflight_seen=max_seen, stages_ms=stages, group_sizes=groups, fp64_tables=fp64,
                           tail=tail)

    def close(self):
        self.pool.shutdown(wait=True)
        self.launchers.shutdown(wait=True)
        for slot in self.slots:  # the workspaces go back to the device
            slot.ws.chunks = []
        torch.cuda.empty_cache()


def main(argv=None) -> int:
    """Serve the seeded mixed-ion request stream once and print the report
    as one JSON line: ``python -m atomx_b200.serve [--requests N]
    [--precision split|fp64] [--offline]``.  ``--offline`` plans every
    request first and hands them all to the server at once (the device's
    capacity on the mix); otherwise they arrive in real time."""
    import argparse
    import json

    from . import workloads as W
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--requests", type=int, default=300)
    ap.add_argument("--precision", default="split", choices=["split", "fp64"])
    ap.add_argument("--slots", type=int, default=2)
    ap.add_argument("--max-group", type=int, default=16)
    ap.add_argument("--offline", action="store_true")
    args = ap.parse_args(argv)
    stream = W.serving_requests(n_requests=args.requests)
    reqs = [Request(rid=i, ion=W.build_ion(spec), k_max=spec.k_max, arrival=t) for i, (t, spec) in enumerate(stream)]
    warm = [Request(rid=-1 - i, ion=W.build_ion(spec), k_max=spec.k_max)
            for i, (_, spec) in enumerate(W.serving_requests(seed=7, n_requests=8))]
    server = SlaterServer(precision=args.precision, max_inflight=args.slots, max_group=args.max_group)
    try:
        server.serve(warm, realtime=False)  # another seed: warms kernels and pools, caches nothing measured
        if args.offline:
            for r in reqs:
                server._plan(r)
            server._plan = lambda r: r  # planned already
        torch.cuda.synchronize()
        rep = server.serve(reqs, realtime=not args.offline)
        torch.cuda.synchronize()
    finally:
        server.close()
    out = rep.summary()
    out.update(offline=args.offline, p99_bound_ms=P99_BOUND_MS,
               errors=[repr(r.error) for r in reqs if r.error is not None][:3])
    print(json.dumps(out))
    return 0 if not out["errors"] else 1


if __name__ == "__main__":
    raise SystemExit(main())
