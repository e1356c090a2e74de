"""Autotuner for batched split-precision tables.

For one batch of ions, each candidate is built and captured as a CUDA graph.
A candidate is a split width in bits (which sets the number of int8 CRT
moduli, the slice count of the Ozaki split), a task order and a row-kernel
layout. The candidate is timed by graph replays with CUDA events, each with
its certificate readback and the FP64 recomputation of the tables that fail
it (a narrow split pays for its recomputed tables), and its tables are
checked against the plain FP64 engine on the same batch. The
checked error is the Schwarz-relative maximum
|R - R_fp64| / sqrt(|R_acac R_bdbd|) over every entry of every table. The
fastest candidate whose error is within ``margin * gate`` wins.

Decisions are cached by the batch's shape key: each ion's (nv, ng, rows, k
set), in order. A batch with the same key reuses the decision without
re-timing.
"""
from __future__ import annotations

import itertools
import time
from dataclasses import dataclass, field

import torch

from .batch import Fp64Batch, SplitBatch

__all__ = ["TuneResult", "autotune_split_batch", "shape_key", "clear_cache"]

_cache: dict = {}


@dataclass
class TuneResult:
    bits: int
    order: str
    fused: object          # None = per-ion default layout, False = two-kernel rows everywhere
    ms: float
    error: float
    trials: list = field(default_factory=list)
    cached: bool = False

    def options(self) -> dict:
        return {"bits": self.bits, "order": self.order, "fused": self.fused}


def shape_key(devs) -> tuple:
    return tuple((d.nv, d.ng, d.plan.n_rows, tuple(d.plan.ks)) for d in devs)


def clear_cache() -> None:
    _cache.clear()


def _max_schwarz_error(batch, ref) -> float:
    worst = 0.0
    for i, dv in enumerate(batch.devs):
        for k in dv.plan.ks:
            a, b = batch.table(i, k), ref.table(i, k)
            dg = torch.diagonal(b).abs().sqrt()
            err = ((a - b).abs() / torch.outer(dg, dg)).max()
            worst = max(worst, float(err))
    return worst


def _time_graph(batch, reps: int) -> float:
    batch.capture()
    batch.replay()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    s = torch.cuda.current_stream()
    # each timed replay includes the certificate's readback and any FP64
    # recomputation it asks for, so a narrower split pays for its escalations
    for a, b in ev:
        a.record(s)
        batch.replay()
        batch.check_status()
        b.record(s)
    torch.cuda.synchronize()
    return min(a.elapsed_time(b) for a, b in ev)


def autotune_split_batch(devs, gate: float = 1e-10, margin: float = 0.5, bits_choices=(32, 34, 36, 38),
                         orders=("lpt", "group"), layouts=(None, False), reps: int = 3,
                         ref: Fp64Batch | None = None) -> TuneResult:
    """Fastest (bits, order, layout) for this batch with error <= margin*gate."""
    key = (shape_key(devs), gate, margin, tuple(bits_choices), tuple(orders), tuple(layouts))
    hit = _cache.get(key)
    if hit is not None:
        return TuneResult(**{**hit.__dict__, "cached": True})
    if ref is None:
        ref = Fp64Batch(devs)
        ref.step()
        torch.cuda.synchronize()
    trials, best = [], None
    for bits, order, fused in itertools.product(bits_choices, orders, layouts):
        t0 = time.perf_counter()
        b = SplitBatch(devs, bits=bits, order=order, fused=fused)
        ms = _time_graph(b, reps)
        err = _max_schwarz_error(b, ref)
        ok = err <= margin * gate
        trials.append({"bits": bits, "n_mod": b.n_mod, "order": order, "fused": fused, "ms": ms, "error": err,
                       "ok": ok, "fp64_tables": len(b.escalated), "tune_s": time.perf_counter() - t0})
        if ok and (best is None or ms < best.ms):
            best = TuneResult(bits=bits, order=order, fused=fused, ms=ms, error=err)
        del b
        torch.cuda.empty_cache()
    if best is None:
        raise RuntimeError(f"no split candidate met {margin} x {gate} on this batch: {trials}")
    best.trials = trials
    _cache[key] = best
    return best
