"""Serving loop for Slater-table requests on one GPU (continuous batching).

A request carries one ion: its radial basis, its spinor coefficients and
kappas, and k_max. This is what an SCF or CI client holds when it asks for
R^k tables. The server runs each request through three stages:

1. host planning, in a worker pool: the pair/row plan and, for the split
   engine, the factored Green operators of the grid and their packed host
   tables (cached by grid content);
2. admission: requests leave the ready queue in arrival order while their
   device footprint fits the HBM budget beside the requests already on the
   GPU, and while a stream slot is free. The footprint is the coefficients,
   orbital values, residue or (g, Y) rows, and the two rotating table
   buffers;
3. device work, on the request's own CUDA stream and set up by the stream
   slot's launcher thread: upload, orbital evaluation, rows, and one
   multipole table after another, each handed to the request's sink with its
   kappa-block ranges (``tables.stream_tables``). An event after the last
   table marks completion. The server polls it, checks the engine's device
   status, frees the request's memory and admits the next one.

Requests that arrive while others are on the GPU are planned at once and
admitted as slots and memory free up. Their kernels then overlap with the
running ones on the device.

Latency is completion minus arrival on the server clock. ``serve`` returns
p50/p99 latency and throughput (ordered R^k entries per second).
Each result is independent of the mix it ran in. The kernels are
deterministic and take no input from other requests, so a request gives the
same tables alone and in a mix; ``tests/test_gpu_serve.py`` checks that.
"""
from __future__ import annotations

import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np
import torch

from .plan import make_plan
from .split import host_tables
from .split_plan import moduli_needed
from .tables import upload_ion

__all__ = ["Request", "ServeReport", "SlaterServer", "ChecksumSink", "footprint_bytes", "P99_BOUND_MS"]

#: The latency bound the loop is held to on the mixed-ion stream (Poisson
#: arrivals at 200 requests/s, Z 2..92, 30..200 B-splines, 10..300 spinors,
#: k_max 2..14): the 99th percentile of (last table delivered - arrival),
#: with two requests on the GPU at once.
P99_BOUND_MS = 500.0


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

    def summary(self) -> dict:
        lat = np.asarray(self.latencies_ms)
        q = np.asarray(self.queue_ms)
        stages = {f"{k}_p50": float(np.percentile(v, 50)) for k, v in self.stages_ms.items() if v}
        return {"requests": self.n, "wall_s": self.wall_s, "entries": self.entries, "stages_ms": stages,
                "throughput_entries_per_s": self.entries / self.wall_s if self.wall_s > 0 else None,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "max_ms": float(lat.max()), "queue_p50_ms": float(np.percentile(q, 50)),
                "queue_p99_ms": float(np.percentile(q, 99)), "precision": self.precision,
                "max_inflight": self.max_inflight_seen}


def footprint_bytes(ion, plan, precision: str) -> int:
    """Device bytes a request holds while it runs (an upper estimate)."""
    nv, ng = ion.bsp["gr"].shape
    n = nv * ng
    n_orb = ion.P.shape[0]
    rows = plan.n_rows
    nmax = max(plan.n_of_k(k) for k in plan.ks)
    base = 8 * (2 * n_orb * n + ion.P.size + ion.Q.size) + 2 * 8 * nmax * nmax + 64 * rows
    if precision == "split":
        kpad = 128 * (-(-((nv - 1) * ng + 64) // 128))
        n_mod = moduli_needed(36, kpad)
        return base + 2 * n_mod * (rows + 128) * kpad + 8 * rows * kpad + 8 * rows * 48
    ld = 32 * (-(-n // 32))
    return base + 2 * 8 * rows * ld


class SlaterServer:
    """Continuous-batching server for R^k table requests on the current GPU."""

    def __init__(self, precision: str = "split", hbm_budget: int | None = None, max_inflight: int = 4,
                 workers: int = 4, bits: int | None = None):
        if precision not in ("split", "fp64"):
            raise ValueError(f"unknown precision {precision!r}")
        self.precision, self.max_inflight, self.bits = precision, int(max_inflight), bits
        if hbm_budget is None:
            free, total = torch.cuda.mem_get_info()
            hbm_budget = int(0.6 * free)
        self.hbm_budget = int(hbm_budget)
        self.device = torch.cuda.current_device()
        self.pool = ThreadPoolExecutor(max_workers=workers)
        # one launcher thread per stream slot: a request's uploads, engine
        # set-up and launches run there, so requests prepare in parallel and
        # the loop itself only admits and retires
        self.launchers = ThreadPoolExecutor(max_workers=self.max_inflight)
        self.streams = [torch.cuda.Stream() for _ in range(self.max_inflight)]

    # ---------------------------------------------------------------- stages
    def _plan(self, req: Request) -> Request:
        t0 = time.perf_counter()
        req.plan = make_plan(req.ion.kappa, req.k_max)
        if self.precision == "split":
            host_tables(np.asarray(req.ion.bsp["gr"], dtype=np.float64).reshape(-1), req.ion.bsp["gr"].shape[1],
                        req.plan.ks)
        req.footprint = footprint_bytes(req.ion, req.plan, self.precision)
        req.entries = req.plan.ordered_entries
        req.timing["plan_ms"] = 1e3 * (time.perf_counter() - t0)
        return req

    def _launch(self, req: Request, stream) -> None:
        from . import tables as T
        req.state["t_launch"] = time.perf_counter()
        sink = req.sink if req.sink is not None else ChecksumSink()
        req.sink = sink
        with torch.cuda.device(self.device), torch.cuda.stream(stream):
            dev = upload_ion(req.ion, k_max=req.k_max, plan=req.plan, stream=stream)
            if self.precision == "split":
                from .split import SplitEngine
                eng = SplitEngine(dev, bits=self.bits, materialize=False)
                eng.stream_tables(sink, stream=stream, check=False)
                req.state["engine"] = eng
            else:
                T.stream_tables(dev, sink, precision="fp64", stream=stream)
            ev = torch.cuda.Event()
            ev.record(stream)
        req.state.update(dev=dev, event=ev, t_enqueued=time.perf_counter())

    def _finish(self, req: Request) -> None:
        st = req.state
        if "t_launch" in st and "t_enqueued" in st:
            req.timing["launch_host_ms"] = 1e3 * (st["t_enqueued"] - st["t_launch"])
            req.timing["after_enqueue_ms"] = 1e3 * (time.perf_counter() - st["t_enqueued"])
        eng = req.state.get("engine")
        try:
            if eng is not None and req.error is None:
                eng.check_status()
        except BaseException as exc:  # a failed request does not stop the server
            req.error = exc
        # buffers allocated on the request's stream return to that stream's
        # pool, so anything a failed launcher enqueued still runs first
        req.state.clear()

    # ------------------------------------------------------------------ loop
    def serve(self, requests: list[Request], realtime: bool = True) -> ServeReport:
        """Run the requests (sorted by arrival) to completion; return timings."""
        todo = deque(sorted(requests, key=lambda r: r.arrival))
        planning, ready, inflight, free_streams = [], deque(), [], list(self.streams)
        used = 0
        max_seen = 0
        t0 = time.perf_counter()

        def now():
            return time.perf_counter() - t0

        while todo or planning or ready or inflight:
            t = now()
            # arrivals: (in real time, or all at once when not realtime)
            while todo and (not realtime or todo[0].arrival <= t):
                r = todo.popleft()
                if not realtime:
                    r.arrival = t
                planning.append((r, self.pool.submit(self._plan, r)))
            # planned requests join the ready queue in arrival order
            still = []
            for r, fut in planning:
                if fut.done():
                    r.planned = now()
                    if fut.exception() is not None:  # e.g. an invalid request
                        r.error, r.done = fut.exception(), r.planned
                    else:
                        ready.append(r)
                else:
                    still.append((r, fut))
            planning = still
            if len(ready) > 1:
                ready = deque(sorted(ready, key=lambda r: r.arrival))
            # completions (a request is done once its launcher has enqueued
            # everything and the completion event has fired)
            for item in list(inflight):
                r, s = item
                fut = r.state.get("launch")
                if fut is not None:
                    if not fut.done():
                        continue
                    del r.state["launch"]
                    if fut.exception() is not None:
                        r.error = fut.exception()
                if r.error is not None or r.state["event"].query():
                    r.done = now()
                    self._finish(r)
                    used -= r.footprint
                    free_streams.append(s)
                    inflight.remove(item)
            # admission by slots and HBM footprint (FIFO; a request larger than
            # the whole budget runs alone)
            while ready and free_streams:
                r = ready[0]
                if inflight and used + r.footprint > self.hbm_budget:
                    break
                ready.popleft()
                s = free_streams.pop()
                r.admitted = now()
                r.state["launch"] = self.launchers.submit(self._launch, r, s)
                used += r.footprint
                inflight.append((r, s))
                max_seen = max(max_seen, len(inflight))
            if not (ready and free_streams):
                time.sleep(2e-4)
        wall = now()
        done = [r for r in requests if r.error is None]
        stages = {k: [r.timing[k] for r in done if k in r.timing]
                  for k in ("plan_ms", "launch_host_ms", "after_enqueue_ms")}
        return ServeReport(n=len(requests), wall_s=wall, entries=int(sum(r.entries for r in done)),
                           latencies_ms=[1e3 * r.latency for r in done],
                           queue_ms=[1e3 * (r.admitted - r.arrival) for r in done], precision=self.precision,
                           max_inflight_seen=max_seen, stages_ms=stages)

    def close(self):
        self.pool.shutdown(wait=True)
        self.launchers.shutdown(wait=True)
