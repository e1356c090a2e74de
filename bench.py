"""Benchmark: R^k integrals/s of whole Slater tables on B200.

Workload (one step = one full table pass on one GPU): the Z=70 ion of 120
order-9 B-splines on [1e-6, 60] bohr with 8 Gauss nodes per cell (N = 896),
200 seeded spinors over kappa = +-1..+-7, every allowed R^k for k = 0..12
(3.18e8 ordered entries).  Inputs are resident on the device before timing;
the ``e2e`` leg starts from host coefficient arrays and ends with the whole
table in pinned host memory.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--engine split|fp64] [--k-max K]
    python bench.py --impl reference   # the reference algorithm on host cores

Multi-GPU: one process per GPU (torchrun); each rank computes its own ion
(same workload, rank-dependent rotation seed) with no data-path collective
(weak scaling); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "R^k integrals/s at <=1e-10 rel vs FP64: split-TC vs plain FP64; serve p50/p99"
UNIT = "integrals/s"
WORKLOAD = "ytterbium_scaleup: Z=70, 120 B-splines order 9, N=896, 200 spinors kappa+-1..+-7, k<=12"


# --------------------------------------------------------------------- helpers
class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    NAMES = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
             0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index: int, period: float = 0.005):
        self.index, self.period = index, period
        self.samples, self.reasons = [], set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._nv = None
            return self
        self._sample()  # one sample at the start of the timed region
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def _sample(self):
        nv = self._nv
        try:
            self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
            bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
            for b, name in self.NAMES.items():
                if bits & b:
                    self.reasons.add(name)
        except Exception:
            pass

    def _run(self):
        while not self._stop.is_set():
            self._stop.wait(self.period)
            self._sample()

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "MEASURED_PEAKS.json"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def dist_setup(n_gpus):
    from atomx_b200 import replicas
    return replicas.init("nccl")


def allreduce_max(x: float, world: int) -> float:
    from atomx_b200 import replicas
    return replicas.reduce_max(x, world)


def allreduce_sum(x: float, world: int) -> float:
    from atomx_b200 import replicas
    return replicas.reduce_sum(x, world)


def barrier(world: int):
    from atomx_b200 import replicas
    replicas.barrier(world)


# ------------------------------------------------------------- CPU baseline
def cpu_baseline(ion, plan, budget_s: float = 12.0, threads: int = 0):
    """Reference-algorithm port (oracle) on the host cores, on a bounded sample.

    Times the two parts of the reference path separately on seeded samples:
    Y^k rows (atomx yk_flat, one per (pair, k) row) and per-entry quadrature
    dots (slater_rk_poisson's sum, one per ordered entry), then extrapolates
    to the whole table: t = rows * t_row + entries * t_dot.
    """
    from oracle import oracle
    bd = ion.bsp
    gr, grw = bd["gr"], bd["grw"]
    nv, ng = gr.shape
    n = nv * ng
    threads = threads or oracle.max_threads()
    rng = np.random.default_rng(99)
    Pg = np.array([oracle.eval_P(c, bd).ravel() for c in ion.P])
    Qg = np.array([oracle.eval_Q(c, bd).ravel() for c in ion.Q])
    nrow = min(plan.n_rows, 4096)
    sel = rng.choice(plan.n_rows, size=nrow, replace=False)
    rho = np.array([Pg[a] * Pg[c] + Qg[a] * Qg[c] for a, c in plan.pairs[plan.row_pair[sel]]])
    ks = plan.row_k[sel]
    t0 = time.perf_counter()
    y = oracle.yk_rows(rho, ks, gr, grw, nv, ng, threads=threads)
    t_rows = time.perf_counter() - t0
    t_row = t_rows / nrow
    g = rho * grw.reshape(1, -1)
    # dots: grow the sample until it takes a good part of the budget
    n_ent = 1 << 16
    spent = t_rows
    t_dot = None
    while True:
        ia = rng.integers(0, nrow, size=n_ent)
        ib = rng.integers(0, nrow, size=n_ent)
        t0 = time.perf_counter()
        oracle.dot_entries(g, y, ia, ib, threads=threads)
        dt = time.perf_counter() - t0
        spent += dt
        t_dot = dt / n_ent
        if dt > budget_s / 3 or spent > budget_s or n_ent >= (1 << 26):
            break
        n_ent *= 4
    total = plan.n_rows * t_row + plan.ordered_entries * t_dot
    return {"value": plan.ordered_entries / total, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"oracle C port of yk_flat + per-entry dot: {nrow} Y^k rows ({t_row*1e6:.1f} us/row) and "
                       f"{n_ent} entries ({t_dot*1e9:.0f} ns/entry) on N={n}, extrapolated to "
                       f"{plan.n_rows} rows + {plan.ordered_entries} entries"),
            "seconds_measured": round(spent, 2)}


REFERENCE_SLICES = 4


def reference_slice(ion, plan, Pg, Qg, phase: int, n_slices: int, threads: int, out_buf=None):
    """One measured slice of the whole table by the reference algorithm.

    The reference path per table entry is atomx's: Y^k of the (bd) density
    (yk_flat, numerics/yk.py:88, computed once per (pair, k) row) and the
    quadrature dot sum_i w_i rho_ac,i Y_i (slater.py:130) per ordered entry.
    Slice ``phase`` of ``n_slices`` takes, in every multipole table, the bd
    rows whose position is ``phase`` mod ``n_slices``, with every ac row of
    that table: the n_slices slices of one table cover it exactly once.
    Returns (ordered entries computed, Y^k rows computed, seconds).
    """
    from oracle import oracle
    bd = ion.bsp
    gr, grw = bd["gr"], bd["grw"]
    nv, ng = gr.shape
    w = grw.reshape(1, -1)
    entries = rows = 0
    t0 = time.perf_counter()
    for k in plan.ks:
        nk = plan.n_of_k(k)
        sel = np.arange(phase, nk, n_slices)
        if sel.shape[0] == 0:
            continue
        pr = plan.pairs[plan.pairs_of_k[k]]
        rho = Pg[pr[:, 0]] * Pg[pr[:, 1]] + Qg[pr[:, 0]] * Qg[pr[:, 1]]
        y = oracle.yk_rows(rho[sel], k, gr, grw, nv, ng, threads=threads)
        g = rho * w
        for c0 in range(0, sel.shape[0], 512):
            yc = y[c0:c0 + 512]
            need = yc.shape[0] * nk
            if out_buf is None or out_buf.size < need:
                out_buf = np.empty(need)
            oracle.dot_block(g, yc, threads=threads, out=out_buf[:need].reshape(yc.shape[0], nk))
        entries += sel.shape[0] * nk
        rows += sel.shape[0]
    return entries, rows, time.perf_counter() - t0


def run_reference(args):
    """--impl reference: the reference algorithm (oracle port) on host cores.

    Every step is measured, not extrapolated: step s computes slice
    s mod 4 of the Z=70 table (a quarter of its entries, every multipole),
    so four consecutive steps compute the whole table once.
    """
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from atomx_b200 import plan as PL
    from atomx_b200 import workloads as W
    from oracle import oracle
    spec = W.ytterbium_scaleup()
    ion = W.build_ion(spec)
    plan = PL.make_plan(ion.kappa, spec.k_max)
    bd = ion.bsp
    Pg = np.array([oracle.eval_P(c, bd).ravel() for c in ion.P])
    Qg = np.array([oracle.eval_Q(c, bd).ravel() for c in ion.Q])
    threads = oracle.max_threads()
    buf = np.empty(512 * max(plan.n_of_k(k) for k in plan.ks))
    times, ents = [], []
    for i in range(args.warmup + args.steps):
        phase = (i - args.warmup) % REFERENCE_SLICES  # the timed steps start at slice 0
        e, _, dt = reference_slice(ion, plan, Pg, Qg, phase, REFERENCE_SLICES, threads, buf)
        if i >= args.warmup:
            times.append(dt)
            ents.append(e)
    total_s = sum(times)
    v = float(sum(ents) / total_s)
    whole = None
    if len(times) >= REFERENCE_SLICES:
        whole = sum(times[:REFERENCE_SLICES])  # four consecutive slices = one whole table
    cb = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
          "sample": (f"measured slices: each step computes 1/{REFERENCE_SLICES} of the Z=70 table "
                     f"(every {REFERENCE_SLICES}th bd row of each multipole against all ac rows; "
                     f"{REFERENCE_SLICES} consecutive steps cover all {plan.ordered_entries} entries): "
                     f"Y^k rows by the oracle C port of yk_flat and one dot per ordered entry"),
          "whole_table_s": whole, "seconds_measured": round(total_s, 2)}
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_s / len(times) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Dirac-Coulomb spinors)",
            "config": {"workload": WORKLOAD, "engine": "reference algorithm (oracle C port), host cores",
                       "k_max": spec.k_max, "entries_per_step": int(statistics.mean(ents)),
                       "unique_entries_per_step": plan.unique_entries // REFERENCE_SLICES,
                       "rows": plan.n_rows, "parallelism": "rank 0 only (host)",
                       "slice": f"1/{REFERENCE_SLICES} of the table per step"},
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- GPU arm
def l2_flush(buf):
    buf.zero_()


def _fp64_engine(dev, stream):
    """Plain FP64 engine: (step, out, workspace)."""
    import torch

    from atomx_b200 import tables as T
    ws = T.Fp64Workspace(dev)
    out = torch.empty(ws.total, device="cuda", dtype=torch.float64)

    def step():
        T.run_fp64(dev, ws, out, stream=stream)
        return out

    return step, out, ws


def _fp64_rows_rate(dev, ws, stream, flush, reps: int = 5) -> dict:
    """The plain engine's Y^k row kernel alone (g and Y^k rows of the whole
    table): CUDA events on the launch stream after an L2 flush, median of
    ``reps``, against the HBM peak.  Algorithmic bytes: the orbital values
    read once and the g and Y rows written."""
    import torch

    from atomx_b200 import _native
    L = _native.load()
    plan = dev.plan
    h = _native.stream_handle(stream)

    def launch():
        _native.check(L.rkb_table_rows_fp64(dev.Pv.data_ptr(), dev.Qv.data_ptr(), dev.n, dev.pairs.data_ptr(),
                                            dev.row_pair.data_ptr(), dev.row_k.data_ptr(), plan.n_rows,
                                            dev.r.data_ptr(), dev.w.data_ptr(), dev.nv, dev.ng, dev.mo.data_ptr(),
                                            dev.mi.data_ptr(), ws.g.data_ptr(), ws.y.data_ptr(), ws.ld, h),
                      "rkb_table_rows_fp64")

    launch()
    ms = float(statistics.median(_time_steps(launch, reps, flush, stream)))
    nbytes = (dev.Pv.numel() + dev.Qv.numel()) * 8 + 2 * plan.n_rows * dev.n * 8
    peaks, src = measured_peaks()
    ach = nbytes / (ms / 1e3) / 1e9
    return {"kernel": "rkb::yk_rows_kernel", "ms": ms, "algorithmic_bytes": int(nbytes), "achieved_gbs": ach,
            "peak_gbs": float(peaks["hbm_gbs"]), "frac": ach / float(peaks["hbm_gbs"]), "peak_source": src,
            "timing": f"CUDA events, L2 flushed, median of {reps} launches"}


def _time_steps(step, n, flush, stream):
    """Device time (ms) of n steps, each after an L2 flush, CUDA events on stream."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
    for a, b in ev:
        l2_flush(flush)
        a.record(stream)
        step()
        b.record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def _fp64_roofline(dev, ws, out, stream, flush):
    """Dominant FP64 kernel (the table contraction) alone, CUDA events on stream."""
    import torch

    from atomx_b200 import _native
    L = _native.load()
    plan = dev.plan
    s = _native.stream_handle(stream)
    _native.check(L.rkb_table_rows_fp64(dev.Pv.data_ptr(), dev.Qv.data_ptr(), dev.n, dev.pairs.data_ptr(),
                                        dev.row_pair.data_ptr(), dev.row_k.data_ptr(), plan.n_rows, dev.r.data_ptr(),
                                        dev.w.data_ptr(), dev.nv, dev.ng, dev.mo.data_ptr(), dev.mi.data_ptr(),
                                        ws.g.data_ptr(), ws.y.data_ptr(), ws.ld, s), "rkb_table_rows_fp64")

    def contract():
        _native.check(L.rkb_table_contract_fp64(ws.g.data_ptr(), ws.y.data_ptr(), ws.ld, ws.ld, ws.row0.data_ptr(),
                                                ws.nk.data_ptr(), ws.out_off.data_ptr(), ws.tasks.data_ptr(),
                                                ws.n_tasks, out.data_ptr(), s), "rkb_table_contract_fp64")

    kms = statistics.median(_time_steps(contract, 3, flush, stream))
    # algorithmic flops: 2*N per unique entry (i <= j) of every table
    flops = 2.0 * dev.n * plan.unique_entries
    peak_tf, src = fp64_peak()
    ach = flops / (kms / 1e3) / 1e12
    return {"bound": "tensor", "achieved": ach, "peak": peak_tf, "unit": "TFLOP/s", "frac": ach / peak_tf,
            "traffic": profiled_traffic("fp64tab::contract_kernel", dev.plan), "kernel": "fp64tab::contract_kernel",
            "kernel_ms": kms, "peak_source": src, "algorithmic_flops": flops, "unit_of_work": "unique entry",
            "units_per_launch": int(plan.unique_entries)}


def _nan_inf(x: float) -> float:
    """A NaN error (a non-finite entry, or 0/0 on a zero diagonal) counts as
    infinite, so that folding with max() cannot drop it."""
    return float("inf") if x != x else x


def table_errors(test, ref, offsets, plan):
    """Errors of a whole table against the FP64 table, per k block.

    schwarz: |x - ref| / sqrt(|ref_ii| |ref_jj|) (the Cauchy-Schwarz scale of
    the entry); floored: |x - ref| / max(|ref|, 1e-6 max|ref| of the k table);
    abs: max |x - ref|.
    """
    import torch
    schwarz = floored = absmax = 0.0
    per_k = {}
    for k in plan.ks:
        nk = plan.n_of_k(k)
        o = offsets[k]
        t = test[o:o + nk * nk].view(nk, nk)
        r = ref[o:o + nk * nk].view(nk, nk)
        d = (t - r).abs()
        dg = r.diagonal().abs().sqrt()
        scale = torch.outer(dg, dg)
        ks_ = _nan_inf(float((d / scale).max()))
        floor = 1e-6 * float(r.abs().max())
        kf = _nan_inf(float((d / r.abs().clamp_min(floor)).max()))
        ka = _nan_inf(float(d.max()))
        per_k[str(k)] = {"schwarz_rel": ks_, "rel_floored_1e-6": kf, "abs": ka}
        schwarz, floored, absmax = max(schwarz, ks_), max(floored, kf), max(absmax, ka)
        del d, scale
    return {"max_schwarz_rel": schwarz, "max_rel_floored_1e-6": floored, "max_abs": absmax, "per_table": per_k}


def profiled_traffic(kernel: str, plan):
    """DRAM bytes per launch of ``kernel`` for this plan, scaled from the
    committed ncu summary (profiles/traffic.json: bytes measured on a smaller
    case and the units it processed); None when no summary is present."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        rec = json.load(f).get(kernel)
    if not rec:
        return None
    return rec["bytes"] / rec["units"] * plan.unique_entries


def run_gpu(args):
    import torch

    from atomx_b200 import tables as T
    from atomx_b200 import workloads as W

    rank, world, local = dist_setup(args.gpus)
    from atomx_b200.replicas import replica_seed
    spec = W.ytterbium_scaleup(seed=replica_seed(2026, rank))
    k_max = spec.k_max if args.k_max is None else args.k_max
    ion = W.build_ion(spec)
    dev = T.upload_ion(ion, k_max=k_max)
    plan = dev.plan
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    engine = args.engine
    if engine == "split":
        from atomx_b200.split import SplitEngine
        eng = SplitEngine(dev)

        def step():
            # check=True: the per-table certificate is read back every step and
            # any table that fails it is recomputed in FP64 inside the step
            return eng.run(stream=stream, upload=False, check=True)

        launches_per_step = eng.launches_per_step
    else:
        step, out64, ws = _fp64_engine(dev, stream)
        launches_per_step = 2

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        t_wall = time.perf_counter()
        if engine == "split":
            eng.kernel_events = []  # the contraction's own launches inside the timed steps
            eng.row_events = []     # and the row kernels
        times = _time_steps(step, args.steps, flush, stream)
        barrier(world)
        t_wall = time.perf_counter() - t_wall
    if engine == "split":
        eng.check_status()
    dev_ms_max = allreduce_max(sum(times), world)
    entries_all = allreduce_sum(float(plan.ordered_entries) * args.steps, world)
    value = entries_all / (dev_ms_max / 1e3)

    extra = {}
    if engine == "split":
        torch.cuda.synchronize()
        live = [a.elapsed_time(b) for a, b in eng.kernel_events]
        rows_live = [a.elapsed_time(b) for a, b in eng.row_events]
        eng.kernel_events = eng.row_events = None
        dom = eng.roofline(kernel_ms=statistics.mean(live))
        peaks, psrc = measured_peaks()
        rms = statistics.mean(rows_live)
        gbs = eng.row_bytes() / (rms / 1e3) / 1e9
        extra["row_kernels"] = {"kernel": f"split rows ({eng.ion_rows.kind})", "ms": rms,
                                "algorithmic_bytes": eng.row_bytes(), "achieved_gbs": gbs,
                                "peak_gbs": float(peaks["hbm_gbs"]), "frac": gbs / float(peaks["hbm_gbs"]),
                                "peak_source": psrc, "bound": "issue (residue arithmetic), HBM below it",
                                "timing": f"CUDA events around the row launches of the {len(rows_live)} timed steps"}
        dom["timing"] = (f"CUDA events on the launch stream around each of the {len(live)} contraction launches "
                         "inside the timed steps (mean)")
        dom["traffic"] = profiled_traffic(dom["kernel"], plan)
        if not args.no_compare:
            # the plain FP64 engine on the same ion: its speed and the split error
            step64, out64, ws = _fp64_engine(dev, stream)
            for _ in range(3):
                step64()
            t64 = _time_steps(step64, max(2, min(args.steps, 5)), flush, stream)
            ms64 = allreduce_max(statistics.mean(t64), world)
            split_out = eng.run(stream=stream, check=True)
            torch.cuda.synchronize()
            err = table_errors(split_out, out64, eng.offsets, plan)
            gate = 1e-10
            extra["fp64_engine"] = {"ms_per_step": ms64, "value": float(plan.ordered_entries) * world / (ms64 / 1e3),
                                    "speedup_split_vs_fp64": ms64 / (dev_ms_max / args.steps),
                                    "row_kernel": _fp64_rows_rate(dev, ws, stream, flush)}
            extra["error_vs_fp64"] = dict(err, gate_schwarz_rel=gate, within_gate=err["max_schwarz_rel"] <= gate)
            del out64, ws
        extra["split"] = eng.info()
    else:
        dom = _fp64_roofline(dev, ws, out64, stream, flush)

    e2e = None if args.no_e2e else e2e_leg(ion, engine, args, world, k_max)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if engine == "fp64" else "i8",
            "data": "synthetic (seeded Dirac-Coulomb spinors, no external dataset)",
            "config": {"workload": WORKLOAD if k_max == spec.k_max else f"{WORKLOAD} (k<={k_max} subset)",
                       "engine": engine, "k_max": k_max, "entries_per_step": plan.ordered_entries,
                       "unique_entries_per_step": plan.unique_entries, "rows": plan.n_rows,
                       "l2": "256 MiB flush between timed steps; working set > L2",
                       "parallelism": f"replicas x{world} (independent ions, no collective)"},
            "roofline": dom, "e2e": e2e, "gpu_launches": launches_per_step * args.steps,
            "clocks": clk.summary(), "wall_s": t_wall}
    line.update(extra)
    # the other workloads (serving, arbitrary grids, the 64-ion batch, the
    # streamed CI table) are measured once, on one GPU: under torchrun every
    # rank would only repeat them while all N GPUs are held
    extra_legs = engine == "split" and world == 1
    if args.serve > 0 and extra_legs:
        line["serve"] = serve_leg(args)
    if not args.no_grid and extra_legs:
        line["grid_yk"] = grid_leg()
    if not args.no_batch and extra_legs:
        line["batch"] = batch_leg()
    if not args.no_stream and extra_legs:
        line["stream"] = stream_leg()
    if not args.no_cell and extra_legs:
        line["cell"] = cell_leg()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:  # the host baseline is measured at N=1 only
        line["cpu_baseline"] = cpu_baseline(ion, plan)
    if rank == 0:
        print(json.dumps(line))
    from atomx_b200 import replicas
    replicas.finalize(world)
    return 0


def fp64_peak():
    """FP64 tensor peak: cuBLAS DGEMM measured here (not in MEASURED_PEAKS)."""
    import torch
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=torch.float64)
    b = torch.randn(n, n, device="cuda", dtype=torch.float64)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = None
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize()
        t = s.elapsed_time(e) / 1e3
        best = t if best is None else min(best, t)
    return 2.0 * n ** 3 / best / 1e12, "measured here: cuBLAS DGEMM 8192^3 (torch.matmul float64), best of 3"


def e2e_leg(ion, engine, args, world, k_max):
    """Same metric through the public API from host arrays to a host table."""
    import torch

    from atomx_b200 import tables as T
    steps = max(1, min(args.steps, 3))
    plan = None
    times = []
    h2d = 0
    for i in range(steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        # host=True, packed=True: each multipole's table (its upper triangle,
        # which holds every ordered entry of the symmetric table) is copied to
        # pinned host memory while the next one is contracted
        tab = T.slater_rk_tables(ion, k_max=k_max, precision=engine, host=True, packed=True)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        assert not tab.values.is_cuda
        plan = tab.plan
        if i > 0:
            times.append(dt)
        h2d = ion.P.nbytes + ion.Q.nbytes
        del tab
    tmax = allreduce_max(float(np.median(times)), world)
    ent = allreduce_sum(float(plan.ordered_entries), world)
    return {"value": ent / tmax, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(plan.unique_entries * 8), "steps": steps,
            "note": "slater_rk_tables(ion, host=True, packed=True) from host coefficients to every table in pinned "
                    "host memory as its packed upper triangle (all ordered entries, R(ac;bd) = R(bd;ac)), "
                    "per-multipole copies overlapped with the contraction"}


def serve_leg(args) -> dict:
    """The seeded Poisson request stream (rate 200/s) served by the
    continuous-batching loop, split engine and plain FP64 engine in turn.

    Each engine's server runs in a process of its own, as a server would
    (``python -m atomx_b200.serve``, on this GPU, while this process waits):
    it warms up on eight requests of another seed, then serves the stream in
    real time and prints its report.  Served inside this process instead,
    after the legs above, some runs stalled for a large fraction of a second
    with the same code."""
    import subprocess

    from atomx_b200 import workloads as W
    from atomx_b200.serve import P99_BOUND_MS
    stream = W.serving_requests(n_requests=args.serve)
    out = {"requests": len(stream), "rate_per_s": 200.0, "arrival_span_s": stream[-1][0],
           "sink": "device: per-(k, row) sums of every multipole table",
           "p99_bound_ms": P99_BOUND_MS,
           "note": "latency = last table delivered - arrival (server clock), realtime Poisson arrivals; "
                   "requests ready together run as one group (one batched contraction launch) in one of "
                   f"{args.serve_slots} stream slots; each engine's server in its own process "
                   "(python -m atomx_b200.serve), warmed up on 8 requests of another seed"}
    torch_sync()
    import torch
    torch.cuda.empty_cache()  # this process's cached device memory back to the server process
    for precision in ("split", "fp64"):
        cmd = [sys.executable, "-m", "atomx_b200.serve", "--requests", str(args.serve), "--precision", precision,
               "--slots", str(args.serve_slots)]
        proc = subprocess.run(cmd, capture_output=True, text=True, cwd=ROOT, timeout=900)
        try:
            rep = json.loads(proc.stdout.strip().splitlines()[-1])
        except (IndexError, ValueError):
            out[precision] = {"error": f"server exited {proc.returncode}: {proc.stderr.strip()[-300:]}"}
            continue
        rep.pop("offline", None)
        rep.pop("p99_bound_ms", None)
        errs = rep.pop("errors", [])
        if errs:
            rep["errors"] = errs
        rep["within_p99_bound"] = rep["p99_ms"] <= P99_BOUND_MS
        out[precision] = rep
    return out


def grid_leg(rows: int = 4000, n: int = 20000, reps: int = 5) -> dict:
    """Arbitrary-grid trapezoid Y^k batch (atomx quadrature.yk_pair_dot_batch_on_grid):
    seeded waves on a geometric grid of n points, `rows` pair rows with ranks
    0..16 and two consumers each, i_cut = n - 1.  Device time per batch (CUDA
    events, inputs resident), against the oracle port of the reference's
    serial kernel on a bounded sample of rows on the host cores."""
    import torch

    from atomx_b200 import _native
    from atomx_b200.quadrature import GridTables
    from oracle import oracle
    rng = np.random.default_rng(77)
    r = np.geomspace(1e-4, 80.0, n)
    env = np.exp(-r / 10.0)
    nw = 32
    P = rng.normal(size=(nw, n)) * env
    Q = 0.02 * rng.normal(size=(nw, n)) * env
    a, b = rng.integers(0, nw, rows), rng.integers(0, nw, rows)
    ks = rng.integers(0, 17, rows)
    ok = np.ones(rows, dtype=bool)
    ptr = np.arange(0, 2 * rows + 1, 2)
    cons = rng.integers(0, 8, 2 * rows)
    W = rng.normal(size=(8, n)) * env
    dev = torch.device("cuda")
    tab = GridTables.get(r, 16, dev)
    d = {k_: torch.as_tensor(v, device=dev) for k_, v in
         dict(P=P, Q=Q, a=a, b=b, k=ks, ok=ok.astype(np.uint8), ptr=ptr, cons=cons, W=W).items()}
    val = torch.zeros(2 * rows, dtype=torch.float64, device=dev)
    work_rows = 8 * torch.cuda.get_device_properties(dev).multi_processor_count
    work = torch.empty((work_rows, n), dtype=torch.float64, device=dev)
    L = _native.load()
    s = torch.cuda.current_stream()

    def launch():
        _native.check(L.rkb_grid_pair_dot_batch(d["P"].data_ptr(), d["Q"].data_ptr(), d["P"].data_ptr(),
                                                d["Q"].data_ptr(), n, d["a"].data_ptr(), d["b"].data_ptr(),
                                                d["k"].data_ptr(), d["ok"].data_ptr(), rows, d["W"].data_ptr(), n,
                                                d["ptr"].data_ptr(), d["cons"].data_ptr(), tab.r.data_ptr(), n,
                                                tab.RK.data_ptr(), tab.inverse.data_ptr(), tab.cuts.data_ptr(),
                                                tab.ncuts, tab.transfers.data_ptr(), tab.ntr, n - 1, val.data_ptr(),
                                                work.data_ptr(), work_rows, _native.stream_handle(s)),
                      "rkb_grid_pair_dot_batch")

    for _ in range(3):
        launch()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for e0, e1 in ev:
        e0.record(s)
        launch()
        e1.record(s)
    torch.cuda.synchronize()
    ms = statistics.median(e0.elapsed_time(e1) for e0, e1 in ev)
    # host: the reference algorithm on a sample of rows, all threads
    sample = min(rows, 256)
    t0 = time.perf_counter()
    ref = oracle.yk_pair_dot_batch_on_grid(P, Q, P, Q, a[:sample], b[:sample], ks[:sample], ok[:sample], W,
                                           ptr[:sample + 1], cons[:2 * sample], r)
    cpu_s = (time.perf_counter() - t0) * rows / sample
    err = float(np.max(np.abs(val[:2 * sample].cpu().numpy() - ref)) / (np.abs(ref).max() + 1e-300))
    # algorithmic bytes per row: P_a, P_b, Q_a, Q_b, rk, inverse, r read twice (two scans),
    # y written and read back, the consumer rows read
    bytes_row = 8 * n * (2 * 7 + 2 + 2)
    return {"workload": f"{rows} pair rows, n={n} geometric grid, ranks 0..16, 2 consumers per row",
            "rows_per_s": rows / (ms / 1e3), "ms_per_batch": ms, "cpu_rows_per_s": rows / cpu_s,
            "cpu_cores": oracle.max_threads(), "cpu_sample_rows": sample,
            "speedup_vs_cpu": cpu_s / (ms / 1e3), "max_rel_err_vs_oracle": err,
            "algorithmic_gbs": bytes_row * rows / (ms / 1e3) / 1e9}


def stream_leg(reps: int = 2) -> dict:
    """The Z=54 CI table (N=2112 with 11 Gauss nodes per cell, 300 spinors,
    k <= 16: 1.95e9 ordered entries, 15.6 GB as FP64) streamed multipole by
    multipole to a device sink that reduces every table (per-row sums), split
    and FP64 in turn; the engine never holds the whole table.  CUDA events
    around each whole stream on the launching stream."""
    import torch

    from atomx_b200 import tables as T
    from atomx_b200 import workloads as W
    from atomx_b200.serve import ChecksumSink
    spec = W.xenon_ci_table()
    dev = T.upload_ion(W.build_ion(spec))
    entries = dev.plan.ordered_entries
    s = torch.cuda.current_stream()
    out = {"workload": "xenon_ci_table: Z=54, 200 B-splines order 9, n_gauss=11 (N=2112), 300 spinors "
                       "kappa+-1..+-9, k<=16", "entries": entries, "table_bytes": entries * 8,
           "sink": "device: per-row sums of every multipole table"}
    for precision in ("split", "fp64"):
        ts, held, info = [], 0, {}
        for i in range(reps + 1):
            sink = ChecksumSink()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            summary = T.stream_tables(dev, sink, precision=precision, stream=s)
            e1.record(s)
            torch.cuda.synchronize()
            if i:
                ts.append(e0.elapsed_time(e1))
            held, info = summary.device_bytes, summary.info
        ms = statistics.median(ts)
        out[precision] = {"ms": ms, "integrals_per_s": entries / (ms / 1e3), "engine_device_bytes": held}
        if precision == "split":
            out[precision]["fp64_multipoles"] = info.get("fp64_multipoles")
            out[precision]["bits"], out[precision]["rows_kernel"] = info.get("bits"), info.get("rows_kernel")
        torch.cuda.empty_cache()
    out["speedup_split_vs_fp64"] = out["fp64"]["ms"] / out["split"]["ms"]
    out.update(stream_diagnostics(dev, s))
    return out


def stream_diagnostics(dev, s) -> dict:
    """One more streamed pass of each engine, instrumented (not the timed
    passes): the split table's error against the plain FP64 table for every
    multipole (Schwarz-relative, floored-relative, absolute), the
    contraction's int8 tensor-pipe rate from CUDA events around each of its
    launches, and the row kernels' algorithmic HBM rate."""
    import torch

    from atomx_b200 import tables as T
    from atomx_b200.split import SplitEngine
    plan = dev.plan
    ref = {}

    def keep(k, table, blocks, stream):
        with torch.cuda.stream(stream):
            ref[k] = table.clone()

    T.stream_tables(dev, keep, precision="fp64", stream=s)
    torch.cuda.synchronize()
    errs = {}

    def compare(k, table, blocks, stream):
        with torch.cuda.stream(stream):
            r = ref[k]
            d = (table - r).abs()
            dg = r.diagonal().abs().sqrt()
            floor = 1e-6 * float(r.abs().max())
            errs[str(k)] = {"schwarz_rel": _nan_inf(float((d / torch.outer(dg, dg)).max())),
                            "rel_floored_1e-6": _nan_inf(float((d / r.abs().clamp_min(floor)).max())),
                            "abs": _nan_inf(float(d.max()))}

    eng = SplitEngine(dev, materialize=False)
    eng.kernel_events, eng.row_events = [], []
    eng.stream_tables(compare, stream=s)
    torch.cuda.synchronize()
    del ref
    torch.cuda.empty_cache()
    ops = ms = 0.0
    for a, b, k in eng.kernel_events:
        ms += a.elapsed_time(b)
        ops += eng.int8_ops([k])[0]
    rms = sum(a.elapsed_time(b) for a, b in eng.row_events)
    peaks, src = measured_peaks()
    tops = ops / (ms / 1e3) / 1e12
    gbs = eng.row_bytes() / (rms / 1e3) / 1e9
    return {"error_vs_fp64": {"max_schwarz_rel": max(e["schwarz_rel"] for e in errs.values()),
                              "max_rel_floored_1e-6": max(e["rel_floored_1e-6"] for e in errs.values()),
                              "max_abs": max(e["abs"] for e in errs.values()), "per_table": errs,
                              "tables_recomputed_fp64": list(eng.escalated)},
            "contraction": {"kernel": eng.dominant_kernel, "ms": ms, "int8_tops": tops,
                            "peak_tops": 2.0 * float(peaks["bf16_tflops"]),
                            "frac": tops / (2.0 * float(peaks["bf16_tflops"])), "peak_source": src,
                            "timing": "CUDA events around each multipole's contraction launch"},
            "row_kernels": {"kind": eng.ion_rows.kind, "ms": rms, "algorithmic_bytes": eng.row_bytes(),
                            "achieved_gbs": gbs, "frac_of_hbm": gbs / float(peaks["hbm_gbs"])}}


def cell_leg(reps: int = 3, cpu_keys: int = 256) -> dict:
    """The cell (bank) engine of atomx convol.py on the Z=70 ion: every
    allowed R^k(ac;bd), k <= 12, as whole cell tables (3.18e8 ordered
    entries; the banks are built once and stay on the device).  CUDA events
    around each whole pass; the FP64 GEMMs are timed against cuBLAS DGEMM.
    Host baseline: the oracle's cell integral (the reference's full-bank
    path, bit-identical to atomx) on a sample of keys, one key per host
    thread (ctypes releases the interpreter lock in the C loops)."""
    from concurrent.futures import ThreadPoolExecutor

    import torch

    from atomx_b200 import convol as C
    from atomx_b200 import workloads as W
    from oracle import cell as OC
    from oracle import oracle
    spec = W.ytterbium_scaleup()
    ion = W.build_ion(spec)
    bd = ion.bsp
    cache = C.ConvolCache(bd)
    cache.release_shared_banks()
    s = torch.cuda.current_stream()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for k in range(spec.k_max + 1):
        cache.bank(k, s)
    e1.record(s)
    torch.cuda.synchronize()
    bank_ms = e0.elapsed_time(e1)
    P = C._stack(list(ion.P), bd["ns"], torch.device("cuda"))
    Q = C._stack(list(ion.Q), bd["ns"], torch.device("cuda"))
    tab = C.cell_tables(P, Q, ion.kappa, bd, spec.k_max, cache=cache)
    plan = tab.plan
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        tab = C.cell_tables(P, Q, ion.kappa, bd, spec.k_max, cache=cache, plan=plan)
        b.record(s)
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    ms = statistics.median(ts)
    kdim = cache.bank(0).kdim
    flops = sum(2.0 * plan.n_of_k(k) * kdim * kdim + 2.0 * kdim * plan.n_of_k(k) * (plan.n_of_k(k) + 1) / 2
                for k in plan.ks)
    peak, psrc = fp64_peak()
    # host: the reference algorithm's cell integral on a seeded sample of keys
    rng = np.random.default_rng(5)
    keys = []
    for _ in range(cpu_keys):
        k = int(rng.choice(plan.ks))
        pk = plan.pairs[plan.pairs_of_k[k]]
        (a_, c_), (b_, d_) = pk[rng.integers(len(pk))], pk[rng.integers(len(pk))]
        keys.append((int(a_), int(c_), int(b_), int(d_), k))
    banks = OC.Banks(bd)
    for k in sorted({kk[4] for kk in keys}):
        for it in OC.ITYPES:
            banks(k, it)
    threads = oracle.max_threads()
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        ref = list(ex.map(lambda kk: OC.slater_rk_cell(ion.P[kk[0]], ion.Q[kk[0]], ion.P[kk[1]], ion.Q[kk[1]],
                                                        ion.P[kk[2]], ion.Q[kk[2]], ion.P[kk[3]], ion.Q[kk[3]],
                                                        bd, kk[4], banks), keys))
    cpu_s = time.perf_counter() - t0
    got = np.array([tab.entry(kk[4], (kk[0], kk[1]), (kk[2], kk[3])) for kk in keys])
    err = float(np.max(np.abs(got - np.array(ref))) / np.max(np.abs(ref)))
    return {"workload": "ytterbium_scaleup cell tables: every allowed R^k(ac;bd), k<=12, by the bank engine "
                        "(atomx convol.py), 120 B-splines order 9 (kdim 2048)",
            "entries": plan.ordered_entries, "ms": ms, "integrals_per_s": plan.ordered_entries / (ms / 1e3),
            "bank_build_ms_k0_12": bank_ms,
            "roofline": {"bound": "tensor (FP64 DMMA)", "achieved_tflops": flops / (ms / 1e3) / 1e12,
                         "peak_tflops": peak, "frac": flops / (ms / 1e3) / 1e12 / peak, "peak_source": psrc,
                         "algorithmic_flops": flops},
            "cpu_baseline": {"value": cpu_keys / cpu_s, "unit": "integrals/s", "cores": threads, "kind": "port",
                             "sample": f"{cpu_keys} seeded keys through the oracle's full-bank cell integral"},
            "speedup_vs_cpu": (plan.ordered_entries / (ms / 1e3)) / (cpu_keys / cpu_s),
            "max_rel_err_vs_oracle": err}


def batch_leg(reps: int = 3) -> dict:
    """The 64-ion uneven batch (Z 20..83, 40..160 B-splines of order 7 or 9,
    20..150 spinors, k_max = 12): every table of every ion in one persistent
    contraction launch, captured with the row launches and the certificate as
    one CUDA graph.  A replay is timed with its certificate readback and the
    FP64 recomputation of the tables that fail it; the split width and task
    order come from the autotuner under the FP64 error gate."""
    import torch

    from atomx_b200 import autotune
    from atomx_b200 import workloads as W
    from atomx_b200.batch import Fp64Batch, SplitBatch
    from atomx_b200.tables import upload_ion
    devs = [upload_ion(W.build_ion(spec)) for spec in W.uneven_batch()]
    entries = sum(d.plan.ordered_entries for d in devs)
    s = torch.cuda.current_stream()

    def timed(batch):
        batch.capture()
        batch.replay()
        batch.check_status()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            batch.replay()
            batch.check_status()
            e1.record(s)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    fp = Fp64Batch(devs)
    ms64 = timed(fp)
    t0 = time.perf_counter()
    tune = autotune.autotune_split_batch(devs, bits_choices=(36, 38), orders=("lpt", "group"), layouts=(None,),
                                         ref=fp)
    tune_s = time.perf_counter() - t0
    del fp
    torch.cuda.empty_cache()
    sb = SplitBatch(devs, **tune.options())
    ms = timed(sb)
    info = sb.info()
    return {"workload": "uneven batch: 64 ions (Z 20..83, ns 40..160, order 7/9, 20..150 spinors, k_max=12)",
            "entries": entries, "split_ms": ms, "split_integrals_per_s": entries / (ms / 1e3),
            "fp64_ms": ms64, "fp64_integrals_per_s": entries / (ms64 / 1e3), "speedup_split_vs_fp64": ms64 / ms,
            "launches_per_replay": sb.launches_per_step, "graph": "one CUDA graph per engine",
            "tables": len(sb.group_of), "fp64_tables": len(info["fp64_tables"]),
            "autotune": {"chosen": tune.options(), "error_vs_fp64": tune.error, "tune_s": tune_s,
                         "trials": [{k_: t[k_] for k_ in ("bits", "n_mod", "order", "ms", "error", "ok")}
                                    for t in tune.trials]},
            "split": {k_: info[k_] for k_ in ("bits", "n_mod", "kpad", "tasks", "rows", "row_kernels")}}


def torch_sync():
    import torch
    torch.cuda.synchronize()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--engine", default=os.environ.get("RKB_ENGINE", "split"), choices=["split", "fp64"])
    ap.add_argument("--k-max", type=int, default=None, help="multipole cut (default: the workload's 12)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64-engine comparison leg")
    ap.add_argument("--serve", type=int, default=300, help="requests in the serving leg (0 = skip)")
    ap.add_argument("--serve-slots", type=int, default=2, help="request groups on the GPU at once in the serving leg")
    ap.add_argument("--no-grid", action="store_true", help="skip the arbitrary-grid Y^k leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-ion batch leg")
    ap.add_argument("--no-stream", action="store_true", help="skip the streamed Z=54 CI table leg")
    ap.add_argument("--no-cell", action="store_true", help="skip the cell (bank) engine leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
