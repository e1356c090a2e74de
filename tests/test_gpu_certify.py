"""Per-table certificate of the split engine and its FP64 recomputation.

Ions of the seeded uneven batch with wide origin cells (first body node near
1e-5, cell ratios near 60) have multipole tables in which atomx's core-cell
self term cancels most of the body energy (g0^T G_00 g0 near -R_body): there
|[X|Z]|^2 exceeds R_aa by up to ~2e3 and no int8 split width reaches the
1e-10 gate.  Every row kernel records |[X|Z]| and the FP64 diagonal R_aa; the
certificate kernel turns them into a per-table error estimate, and tables
over the limit are recomputed by the FP64 engine.  Checked here:
- the row record and the estimate against the CPU emulation (all three row
  kernels);
- one ion, materialised and streamed: the cancelling table goes to FP64 and
  every table is within the gate of the plain FP64 engine;
- the whole 64-ion uneven batch (one graph replay) within the gate.
"""
import numpy as np
import pytest

from oracle import oracle
from split_emulation import transform_rows, unpack_table

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GATE = 1e-10
CANCELLING_ION, CANCELLING_K = 42, 7   # |[X|Z]|^2 / R_aa ~ 2.5e3


def _schwarz(a, ref):
    d = torch.diagonal(ref).abs().sqrt()
    return float(((a - ref).abs() / torch.outer(d, d)).max())


def _ion(index):
    from atomx_b200 import workloads as W
    from atomx_b200.tables import upload_values
    spec = W.uneven_batch()[index]
    ion = W.build_ion(spec)
    bd = ion.bsp
    Pg = np.array([oracle.eval_P(c, bd).ravel() for c in ion.P])
    Qg = np.array([oracle.eval_Q(c, bd).ravel() for c in ion.Q])
    return ion, Pg, Qg, upload_values(Pg, Qg, ion.kappa, bd["gr"], bd["grw"], spec.k_max)


@pytest.fixture(scope="module")
def cancelling():
    return _ion(CANCELLING_ION)


@pytest.mark.parametrize("rows_kernel", ["two", "fused", "cells"])
def test_row_record_and_certificate_match_emulation(cancelling, rows_kernel):
    from atomx_b200.split import CB_STRIDE, SplitEngine
    ion, Pg, Qg, dev = cancelling
    eng = SplitEngine(dev, rows_kernel=rows_kernel)
    eng.rows()
    torch.cuda.synchronize()
    plan = dev.plan
    nv, ng = ion.bsp["gr"].shape
    cb = eng.cbound.cpu().numpy()
    rs = eng.rowscale.cpu().numpy()
    est = eng.est.cpu().numpy()
    assert cb.shape[1] == CB_STRIDE
    flat, koff = eng.ktab.cpu().numpy(), eng.koff.cpu().numpy()
    for gi, k in enumerate(plan.ks):
        F = unpack_table(flat, int(koff[k]), nv, ng)
        off, nk = plan.k_row_offset[k], plan.n_of_k(k)
        rows = np.arange(off, off + nk)
        rho = np.array([Pg[a] * Pg[c] + Qg[a] * Qg[c] for a, c in plan.pairs[plan.row_pair[rows]]])
        g = rho * ion.bsp["grw"].reshape(1, -1)
        X, Z, lf, rt = transform_rows(g, F, nv, ng)
        nrm = np.sqrt((X * X).sum(1) + (Z * Z).sum(1))
        raa = (X * X).sum(1) - (Z * Z).sum(1) + (lf * rt).sum(1)
        np.testing.assert_allclose(cb[rows, 4], nrm, rtol=1e-12)
        assert np.all(np.abs(cb[rows, 5] - raa) <= 1e-12 * nrm ** 2), k
        assert np.all(cb[rows, 6:] == 0.0)
        # the estimate from the device's own record
        live = cb[rows, 4] > 0
        rd = np.sqrt(np.abs(cb[rows, 5]))[live]
        ref = (rs[rows][live] / rd).max() * (cb[rows, 4][live] / rd).max()
        assert est[gi] == pytest.approx(ref, rel=1e-12), k
    ks = list(plan.ks)
    assert not est[ks.index(CANCELLING_K)] <= eng.cert_limit
    flagged = int(eng.status[1].item())
    assert flagged == int(np.sum(~(est <= eng.cert_limit))) >= 1


def test_cell_kernel_with_more_than_64_z_columns():
    """Ion 43 (nv 98, ng 9, up to 65 Z columns) runs on the cell kernel: its
    residues rebuild [X | Z] to the rounding quantum and B negates Z."""
    from atomx_b200.split import SplitEngine
    from split_emulation import crt_exact
    ion, Pg, Qg, dev = _ion(43)
    eng = SplitEngine(dev)
    assert eng.ion_rows.kind == "cells" and eng.max_z > 64
    eng.rows()
    torch.cuda.synchronize()
    plan = dev.plan
    nv, ng = ion.bsp["gr"].shape
    resA = eng.resA.cpu().numpy().astype(np.int64)
    resB = eng.resB.cpu().numpy().astype(np.int64)
    rs = eng.rowscale.cpu().numpy()
    flat, koff = eng.ktab.cpu().numpy(), eng.koff.cpu().numpy()
    rng = np.random.default_rng(43)
    for k in plan.ks:
        if eng.nz[k] <= 64:
            continue
        F = unpack_table(flat, int(koff[k]), nv, ng)
        off, nk = plan.k_row_offset[k], plan.n_of_k(k)
        rows = np.sort(rng.choice(nk, size=min(12, nk), replace=False)) + off
        rho = np.array([Pg[a] * Pg[c] + Qg[a] * Qg[c] for a, c in plan.pairs[plan.row_pair[rows]]])
        X, Z, _, _ = transform_rows(rho * ion.bsp["grw"].reshape(1, -1), F, nv, ng)
        ref = np.concatenate([X, Z], axis=1)
        pos = eng.column_positions(k)
        got = crt_exact([resA[i][rows][:, pos] for i in range(eng.n_mod)], eng.moduli) * rs[rows][:, None]
        assert np.all(np.abs(got - ref) <= (0.5 + 1e-6) * rs[rows][:, None] + 1e-15 * np.abs(ref)), k
        zpos = pos[X.shape[1]:]
        xb = crt_exact([resB[i][rows][:, zpos] for i in range(eng.n_mod)], eng.moduli)
        xa = crt_exact([resA[i][rows][:, zpos] for i in range(eng.n_mod)], eng.moduli)
        np.testing.assert_array_equal(xb, -xa)
        break
    else:
        pytest.fail("no multipole with more than 64 Z columns")


def test_single_ion_recomputes_failing_tables_in_fp64(cancelling):
    from atomx_b200.split import SplitEngine
    from atomx_b200.tables import tables_for
    ion, Pg, Qg, dev = cancelling
    eng = SplitEngine(dev)
    out = eng.run(check=True)
    torch.cuda.synchronize()
    assert CANCELLING_K in eng.escalated and eng.info()["fp64_multipoles"] == eng.escalated
    assert len(eng.escalated) < len(dev.plan.ks)  # the others stay on the split path
    plain = tables_for(dev, "fp64")
    for k in dev.plan.ks:
        nk = dev.plan.n_of_k(k)
        a = out[eng.offsets[k]:eng.offsets[k] + nk * nk].view(nk, nk)
        assert _schwarz(a, plain.table(k)) <= GATE, k
        if k in eng.escalated:
            r = plain.table(k)
            assert float((a - r).abs().max()) <= 1e-14 * float(r.abs().max()), k
    # a second run reaches the same decision and the same values
    first = out.clone()
    eng.run(check=True)
    torch.cuda.synchronize()
    assert torch.equal(eng.out, first)


def test_streamed_tables_take_the_same_fp64_route(cancelling):
    from atomx_b200.split import SplitEngine
    from atomx_b200.tables import HostTableSink, tables_for
    ion, Pg, Qg, dev = cancelling
    sink = HostTableSink()
    eng = SplitEngine(dev, materialize=False)
    eng.stream_tables(sink, check=True)
    tabs = sink.wait()
    assert CANCELLING_K in eng.escalated
    plain = tables_for(dev, "fp64")
    for k in dev.plan.ks:
        assert _schwarz(tabs[k].cuda(), plain.table(k)) <= GATE, k


def test_uneven_batch_of_64_ions_within_gate():
    """Every table of all 64 ions (1.45e9 entries) in one graph replay."""
    from atomx_b200 import workloads as W
    from atomx_b200.batch import Fp64Batch, SplitBatch
    from atomx_b200.tables import upload_ion
    devs = [upload_ion(W.build_ion(s)) for s in W.uneven_batch()]
    ref = Fp64Batch(devs)
    ref.step()
    b = SplitBatch(devs)
    b.replay()
    b.check_status()
    torch.cuda.synchronize()
    worst = 0.0
    for i, dv in enumerate(devs):
        for k in dv.plan.ks:
            worst = max(worst, _schwarz(b.table(i, k), ref.table(i, k)))
    assert worst <= GATE, worst
    groups = len(b.group_of)
    assert 1 <= len(b.escalated) <= groups // 10, b.escalated
    assert (CANCELLING_ION, CANCELLING_K) in b.escalated


def test_deferred_certificate_redelivers_the_fp64_table(cancelling):
    """A sink that keeps one table per multipole (replaces_tables) is served
    without the mid-stream wait for the certificate: every table is
    contracted at once and check_status() hands the failing table to the
    sink again, recomputed in FP64.  Its final tables equal those of a sink
    served the strict way (the certificate read before any contraction)."""
    from atomx_b200.split import SplitEngine

    class Keep:
        def __init__(self, replaces):
            self.replaces_tables = replaces
            self.tables, self.calls = {}, []

        def __call__(self, k, table, blocks, stream):
            with torch.cuda.stream(stream):
                self.tables[k] = table.clone()
            self.calls.append(k)

    ion, Pg, Qg, dev = cancelling
    strict, lazy = Keep(False), Keep(True)
    SplitEngine(dev, materialize=False).stream_tables(strict, check=True)
    eng = SplitEngine(dev, materialize=False)
    eng.stream_tables(lazy, check=True)
    torch.cuda.synchronize()
    assert CANCELLING_K in eng.escalated
    assert strict.calls == list(dev.plan.ks)
    assert lazy.calls == list(dev.plan.ks) + list(eng.escalated)
    for k in dev.plan.ks:
        assert torch.equal(strict.tables[k], lazy.tables[k]), k
