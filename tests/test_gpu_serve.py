"""Serving loop: continuous batching of Slater-table requests on one GPU.

A seeded Poisson stream of small requests (the serving workload's ranges,
clipped so the test stays short) runs through the server in one group, in
several groups in flight at once, and then each request alone. Every table of
every request must be identical in all runs, since no request's work depends
on another's. The report carries p50/p99 latency, throughput and the group
sizes.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


class _Collect:
    def __init__(self):
        self.tables = {}

    def __call__(self, k, table, blocks, stream):
        with torch.cuda.stream(stream):
            self.tables[k] = table.clone()


def _requests(n=10, seed=4200):
    from atomx_b200 import workloads as W
    from atomx_b200.serve import Request
    stream = W.serving_requests(seed=seed, n_requests=n, max_ns=90, max_orbitals=60, max_kmax=6)
    return [(Request(rid=i, ion=W.build_ion(spec), k_max=spec.k_max, arrival=t), spec)
            for i, (t, spec) in enumerate(stream)]


@pytest.mark.parametrize("precision", ["split", "fp64"])
def test_results_alone_equal_results_in_the_mix(precision):
    """Every request in one group of ten (one contraction launch), in groups
    of three on four slots at once, and alone: identical tables."""
    from atomx_b200.serve import Request, SlaterServer
    runs = []
    for max_group in (16, 3):
        reqs = [r for r, _ in _requests()]
        for r in reqs:
            r.sink = _Collect()
        server = SlaterServer(precision=precision, max_inflight=4, max_group=max_group)
        rep = server.serve(reqs, realtime=False)  # all at once: the mix is as dense as it gets
        server.close()
        torch.cuda.synchronize()
        assert all(r.error is None for r in reqs), [r.error for r in reqs]
        assert rep.max_inflight_seen > 1
        summ = rep.summary()
        assert summ["p99_ms"] >= summ["p50_ms"] > 0 and summ["throughput_entries_per_s"] > 0
        assert rep.group_sizes == ([10] if max_group == 16 else [3, 3, 3, 1]), rep.group_sizes
        runs.append(reqs)
    alone_server = SlaterServer(precision=precision, max_inflight=1)
    for i, r in enumerate(runs[0]):
        solo = Request(rid=r.rid, ion=r.ion, k_max=r.k_max, sink=_Collect())
        alone_server.serve([solo], realtime=False)
        torch.cuda.synchronize()
        for mix in runs:
            tabs = mix[i].sink.tables
            assert sorted(solo.sink.tables) == sorted(tabs)
            for k, t in tabs.items():
                assert torch.equal(t, solo.sink.tables[k]), (r.rid, k)
    alone_server.close()


def test_streamed_request_agrees_with_its_grouped_run():
    """A request above group_bytes runs alone on the streaming engine; its
    tables agree with the grouped run to the split's rounding (both are
    within the split gate of the FP64 engine)."""
    from atomx_b200.serve import Request, SlaterServer
    (r, _), = _requests(n=1, seed=4204)
    r.sink = _Collect()
    grouped = SlaterServer(precision="split", max_inflight=1)
    grouped.serve([r], realtime=False)
    grouped.close()
    s = Request(rid=0, ion=r.ion, k_max=r.k_max, sink=_Collect())
    streamed = SlaterServer(precision="split", max_inflight=1, group_bytes=1)
    rep = streamed.serve([s], realtime=False)
    streamed.close()
    torch.cuda.synchronize()
    assert s.error is None and r.error is None and rep.group_sizes == [1]
    assert sorted(s.sink.tables) == sorted(r.sink.tables)
    for k, t in r.sink.tables.items():
        u = s.sink.tables[k]
        d = torch.diagonal(t).abs().sqrt()
        assert float(((t - u).abs() / torch.outer(d, d)).max()) <= 1e-10, k


def test_realtime_stream_reports_latency_and_admits_by_memory():
    from atomx_b200.serve import SlaterServer
    reqs = [r for r, _ in _requests(n=16, seed=4201)]
    fp = sorted(r.footprint for r in reqs)
    server = SlaterServer(precision="split", max_inflight=4)
    rep = server.serve(reqs)
    assert all(r.error is None for r in reqs)
    assert all(r.done >= r.admitted >= r.arrival for r in reqs)
    s = rep.summary()
    assert s["requests"] == 16 and s["p50_ms"] > 0
    # a budget that fits one request at a time serialises the device work
    reqs2 = [r for r, _ in _requests(n=6, seed=4202)]
    small = SlaterServer(precision="split", max_inflight=4, hbm_budget=1)
    rep2 = small.serve(reqs2, realtime=False)
    assert rep2.max_inflight_seen == 1 and all(r.error is None for r in reqs2)
    server.close()
    small.close()


class _Replacing(_Collect):
    """A sink that keeps one table per multipole: the server delivers every
    table without waiting for the certificate and delivers a table that
    failed it again, recomputed in FP64."""
    replaces_tables = True


@pytest.mark.parametrize("sink", [_Collect, _Replacing])
@pytest.mark.parametrize("max_group", [16, 1])
def test_served_cancelling_ion_is_within_the_gate(sink, max_group):
    """A request whose k=7 table fails the split certificate (ion 42 of the
    uneven batch) served in a mix, in a group or in a slot of its own: its
    k=7 table takes the FP64 route (before delivery, or delivered again) and
    every table is within 1e-10 (Schwarz-relative) of the FP64 engine."""
    from atomx_b200 import workloads as W
    from atomx_b200.serve import Request, SlaterServer
    from atomx_b200.tables import tables_for, upload_ion
    spec = W.uneven_batch()[42]
    ion = W.build_ion(spec)
    target = Request(rid=99, ion=ion, k_max=spec.k_max, sink=sink())
    others = [r for r, _ in _requests(n=4, seed=4203)]
    for r in others:
        r.sink = sink()
    server = SlaterServer(precision="split", max_inflight=4, max_group=max_group)
    rep = server.serve([target] + others, realtime=False)
    assert rep.fp64_tables >= 1
    torch.cuda.synchronize()
    assert target.error is None and all(r.error is None for r in others)
    plain = tables_for(upload_ion(ion, k_max=spec.k_max), "fp64")
    assert sorted(target.sink.tables) == sorted(plain.ks)
    worst = 0.0
    for k, t in target.sink.tables.items():
        ref = plain.table(k)
        d = torch.diagonal(ref).abs().sqrt()
        worst = max(worst, float(((t - ref).abs() / torch.outer(d, d)).max()))
    assert worst <= 1e-10, worst
    # the cancelling table itself came from the FP64 engine
    assert float((target.sink.tables[7] - plain.table(7)).abs().max()) <= 1e-14 * float(plain.table(7).abs().max())
    server.close()


@pytest.mark.parametrize("name", ["ytterbium_scaleup", "neon_small"])
def test_staged_inputs_equal_uploaded_ones(name):
    """tables.stage_ion (one pinned buffer, one copy, orbitals evaluated into
    the same allocation) gives every array upload_ion gives, and the staged
    factor tables equal the cached device copies; a batch over staged inputs
    gives the same tables as over uploaded ones."""
    from atomx_b200 import workloads as W
    from atomx_b200.batch import SplitBatch
    from atomx_b200.plan import make_plan
    from atomx_b200.split import IonRows, host_tables
    from atomx_b200.tables import stage_ion, upload_ion
    spec = getattr(W, name)()
    ion = W.build_ion(spec)
    plan = make_plan(ion.kappa, spec.k_max)
    H = host_tables(np.asarray(ion.bsp["gr"], dtype=np.float64).reshape(-1), ion.bsp["gr"].shape[1], plan.ks)
    s = torch.cuda.Stream()
    staged, dtab, pinned = stage_ion(ion, plan, s, None, H)
    s.synchronize()
    ref = upload_ion(ion, k_max=spec.k_max, plan=plan)
    torch.cuda.synchronize()
    for f in ("r", "w", "mo", "mi", "Pv", "Qv", "pairs", "row_pair", "row_k"):
        a, b = getattr(staged, f), getattr(ref, f)
        assert a.dtype == b.dtype and torch.equal(a.reshape(-1), b.reshape(-1)), f
    rows_s, rows_r = IonRows(staged, device_tables=dtab), IonRows(ref)
    for f in ("ktab", "koff", "zcount"):
        assert torch.equal(getattr(rows_s, f), getattr(rows_r, f)), f
    assert rows_s.kind == rows_r.kind
    if rows_r.ktab_t is not None:
        assert torch.equal(rows_s.ktab_t, rows_r.ktab_t) and torch.equal(rows_s.koff_t, rows_r.koff_t)
    a = SplitBatch([staged], ion_rows=[rows_s])
    b = SplitBatch([ref], ion_rows=[rows_r])
    a.step()
    b.step()
    a.check_status()
    b.check_status()
    assert torch.equal(a.out, b.out)
    # a second, smaller ion reuses the grown pinned buffer
    small = W.build_ion(W.neon_small())
    p2 = make_plan(small.kappa, 2)
    _, _, pinned2 = stage_ion(small, p2, s, pinned, None)
    assert pinned2 is pinned


def test_command_line_serves_the_stream(capsys):
    """``python -m atomx_b200.serve``: a short run of the seeded stream
    (after its warm-up requests) reports every request served."""
    import json

    from atomx_b200.serve import main
    assert main(["--requests", "6", "--offline"]) == 0
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert out["requests"] == 6 and out["errors"] == [] and out["offline"] is True
    assert out["p99_ms"] >= out["p50_ms"] > 0 and out["throughput_entries_per_s"] > 0
