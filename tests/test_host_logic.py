"""CPU checks of the engines' host logic: task orders, split widths, row
kernel choice, the cell-minor factor layout and the serving footprint."""
import numpy as np
import pytest


def test_batch_tasks_cover_upper_tiles_and_lpt_orders_by_cost():
    from atomx_b200.batch import batch_tasks
    from atomx_b200.tables import tile_tasks
    sizes, costs = [300, 1, 129, 0, 700], [896, 640, 1024, 512, 768]
    ref = tile_tasks(sizes)
    for order in ("group", "lpt"):
        t = batch_tasks(sizes, costs, order)
        assert sorted(map(tuple, t)) == sorted(map(tuple, ref))
        assert np.all(t[:, 2] >= t[:, 1])
    lpt = batch_tasks(sizes, costs, "lpt")
    c = np.asarray(costs)[lpt[:, 0]]
    assert np.all(np.diff(c) <= 0)
    with pytest.raises(ValueError):
        batch_tasks(sizes, costs, "random")


def test_tile_tasks_are_each_groups_upper_triangle_in_order():
    from atomx_b200.tables import tile_tasks
    rng = np.random.default_rng(0)
    for trial in range(60):
        sizes = rng.integers(0, 3000, rng.integers(0, 30)) if trial % 7 else np.zeros(trial % 3, int)
        ref = []
        for g, n in enumerate(sizes):
            ti, tj = np.triu_indices((int(n) + 127) // 128)
            ref += [(g, a, b) for a, b in zip(ti, tj)]
        got = tile_tasks(sizes)
        assert got.dtype == np.int32 and got.shape == (len(ref), 3)
        assert [tuple(map(int, t)) for t in got] == ref


def test_blocked_tile_order_is_a_permutation_by_blocks():
    """tile_tasks(block=b): every group's upper-triangle tiles, groups still
    contiguous and in order, tiles ordered by (block row, block column), then
    row-major inside a block."""
    from atomx_b200.tables import tile_tasks
    rng = np.random.default_rng(5)
    for trial in range(30):
        sizes = rng.integers(0, 4000, rng.integers(1, 12))
        for b in (1, 3, 8):
            base, got = tile_tasks(sizes), tile_tasks(sizes, block=b)
            assert got.shape == base.shape and got.dtype == np.int32
            assert sorted(map(tuple, got)) == sorted(map(tuple, base))
            g = got[:, 0]
            assert np.all(np.diff(g) >= 0)  # groups contiguous, in order
            key = np.stack([g, got[:, 1] // b, got[:, 2] // b, got[:, 1], got[:, 2]], axis=1)
            assert all(tuple(key[i]) < tuple(key[i + 1]) for i in range(len(key) - 1))
    order = [2, 0, 1]
    got = tile_tasks([300, 500, 900], order=order, block=2)
    assert [int(x) for x in dict.fromkeys(got[:, 0])] == order


def test_split_width_choice():
    from atomx_b200.split import KDIM_MAX, check_kdim, choose_width
    from atomx_b200.split_plan import MODULI, bits_for_moduli, moduli_needed
    import math
    for kdim in (128, 896, 1024, 2176, KDIM_MAX):
        bits, n_mod = choose_width(None, None, kdim)
        assert n_mod == moduli_needed(36, kdim) and bits >= 36
        # the chosen width is exact: 2 kdim 2^(2 bits) + 2 < M
        assert 2 * kdim * (1 << (2 * bits)) + 2 < math.prod(MODULI[:n_mod])
        assert bits == max(36, bits_for_moduli(n_mod, kdim))
    assert choose_width(30, None, 896) == (30, moduli_needed(30, 896))
    # fixed moduli: the widest split they hold at each length, and no wider
    assert choose_width(None, 11, 256) == (39, 11) and choose_width(None, 11, KDIM_MAX) == (37, 11)
    with pytest.raises(ValueError):
        choose_width(38, 10, 1024)
    with pytest.raises(ValueError):
        check_kdim(KDIM_MAX + 128)


def test_row_kernel_fit_rules():
    from atomx_b200.split import cells_fit, fused_body_positions, fused_body_width, fused_fits
    assert cells_fit(112, 8, 37) and cells_fit(192, 11, 64) and not cells_fit(200, 11, 64)
    assert cells_fit(98, 9, 65) and cells_fit(120, 9, 128) and not cells_fit(100, 9, 129)
    assert not cells_fit(100, 4, 0) and not cells_fit(100, 12, 0)
    assert fused_fits(112, 8, 37) and not fused_fits(192, 11, 10)
    for nv, ng in [(112, 8), (34, 7), (60, 5), (30, 11)]:
        pos = fused_body_positions(nv, ng)
        assert len(np.unique(pos)) == (nv - 1) * ng and pos.max() < fused_body_width(nv, ng)


def test_cell_minor_tables_are_transposes_of_the_packed_ones():
    from atomx_b200 import workloads as W
    from atomx_b200.split import host_tables
    from atomx_b200.split_plan import factor_table_layout
    ion = W.build_ion(W.neon_small())
    gr = ion.bsp["gr"]
    nv, ng = gr.shape
    H = host_tables(gr.ravel(), ng, [0, 1, 2])
    o = factor_table_layout(nv, ng)
    n = nv * ng
    for k in (0, 1, 2):
        F = H["flat"][H["koff"][k]:]
        T = H["flat_t"][H["koff_t"][k]:]
        u = F[:n].reshape(nv, ng)
        L = F[o["Lb"]:o["Lb"] + nv * ng * ng].reshape(nv, ng, ng)
        C = F[o["C"]:o["C"] + n].reshape(nv, ng)
        np.testing.assert_array_equal(T[:n].reshape(ng, nv), u.T)
        np.testing.assert_array_equal(T[n:2 * n].reshape(ng, nv), C.T)
        np.testing.assert_array_equal(T[2 * n:2 * n + nv * ng * ng].reshape(ng, ng, nv), L.transpose(1, 2, 0))
    assert host_tables(gr.ravel(), ng, [0, 1, 2]) is H  # cached


@pytest.mark.parametrize("name,ks", [("neon_small", (0, 1, 2)), ("ytterbium_scaleup", tuple(range(13))),
                                     ("neon_small", (1, 3, 4))])
@pytest.mark.parametrize("threads", [1, 3])
def test_host_tables_equal_the_per_multipole_factors(name, ks, threads, monkeypatch):
    """host_tables (one native call over all multipoles) equals the
    per-multipole factorisation laid end to end, with the cell-minor copy
    built by transposes, bit for bit, on one host thread or several."""
    from atomx_b200 import split as SP
    from atomx_b200 import workloads as W
    monkeypatch.setattr(SP, "HOST_TABLE_THREADS", threads)
    ion = W.build_ion(getattr(W, name)())
    gr = np.asarray(ion.bsp["gr"], dtype=np.float64)
    nv, ng = gr.shape
    n = nv * ng
    SP._host_cache.clear()
    H = SP.host_tables(gr.ravel(), ng, ks)
    F = SP.factors_for_grid(gr.ravel(), ng, ks)
    assert np.array_equal(H["flat"], np.concatenate([F[k] for k in ks]))
    pos = pos_t = 0
    for k in range(max(ks) + 1):
        if k not in ks:
            assert H["koff"][k] == -1 and H["koff_t"][k] == -1
            continue
        assert H["koff"][k] == pos and np.array_equal(H["factors"][k], F[k])
        Fk = F[k]
        u_ = Fk[:n].reshape(nv, ng).T
        L_ = Fk[n:n + nv * ng * ng].reshape(nv, ng, ng).transpose(1, 2, 0)
        C_ = Fk[n + nv * ng * ng:n + nv * ng * ng + n].reshape(nv, ng).T
        t = np.concatenate([u_.ravel(), C_.ravel(), L_.ravel()])
        assert H["koff_t"][k] == pos_t and np.array_equal(H["flat_t"][pos_t:pos_t + t.shape[0]], t)
        assert H["nz"][k] == int(Fk[n + nv * ng * ng + n + ng + ng * ng + 1])
        pos += Fk.shape[0]
        pos_t += t.shape[0]
    assert H["flat_t"].shape[0] == pos_t
    SP._host_cache.clear()


def test_workspace_views_are_aligned_disjoint_and_merge_on_reset():
    """The reusable batch workspace (exercised on host memory): aligned,
    non-overlapping views of the requested shapes; a batch that outgrows it
    adds a chunk, and reset merges the chunks so the next batch of the same
    size takes no new memory."""
    import torch

    from atomx_b200.batch import Workspace
    ws = Workspace(device=torch.device("cpu"))
    ws.MIN_CHUNK = 4096
    shapes = [((3, 5, 128), torch.int8), ((7,), torch.float64), ((9, 14), torch.float64), ((3000,), torch.float64)]
    for rnd in range(3):
        views = [ws.take(sh, dt) for sh, dt in shapes]
        spans = []
        for v, (sh, dt) in zip(views, shapes):
            assert tuple(v.shape) == sh and v.dtype == dt and v.is_contiguous()
            base = [c.data_ptr() for c in ws.chunks if c.data_ptr() <= v.data_ptr() < c.data_ptr() + c.numel()]
            assert len(base) == 1 and (v.data_ptr() - base[0]) % Workspace.ALIGN == 0  # (device chunks: 512-aligned)
            spans.append((v.data_ptr(), v.data_ptr() + v.numel() * v.element_size()))
            v.fill_(rnd + 1)
        spans.sort()
        assert all(a[1] <= b[0] for a, b in zip(spans, spans[1:]))
        assert all(bool((v == rnd + 1).all()) for v in views)
        ws.reset()
        if rnd == 0:
            merged = ws.capacity
        assert len(ws.chunks) == 1 and ws.capacity == merged
    ws.reserve(3 * merged)
    assert len(ws.chunks) == 1 and ws.capacity == 3 * merged
    ws.take((10,), torch.float64)
    with pytest.raises(RuntimeError):
        ws.reserve(1)


def test_serving_footprint_grows_with_the_request():
    from atomx_b200 import plan as PL
    from atomx_b200 import workloads as W
    from atomx_b200.serve import footprint_bytes
    small = W.build_ion(W.neon_small())
    big = W.build_ion(W.ytterbium_scaleup())
    fs = footprint_bytes(small, PL.make_plan(small.kappa, 2), "split")
    fb = footprint_bytes(big, PL.make_plan(big.kappa, 12), "split")
    ff = footprint_bytes(big, PL.make_plan(big.kappa, 12), "fp64")
    assert 0 < fs < fb and ff > 0
    # the split estimate covers the residue matrices of that ion (11 moduli, two copies)
    assert fb > 2 * 11 * 56209 * 1024
    # held whole (a request in a group), the Z=70 tables add their 2.5 GB
    whole = footprint_bytes(big, PL.make_plan(big.kappa, 12), "split", whole_tables=True)
    assert whole - fb > 8 * 318112753 - 2 * 8 * 14000 ** 2


def _req(rid, fp, streamed=False):
    from atomx_b200.serve import Request
    r = Request(rid=rid, ion=None, k_max=0, arrival=float(rid))
    r.footprint, r.state["streamed"] = fp, streamed
    return r


def test_serving_groups_are_fifo_and_bounded():
    """Group formation of the serving loop (no GPU): arrival order, at most
    max_group requests and group_bytes of device memory, within the HBM
    budget beside the groups in flight, a streamed request alone, and the
    first request of an idle device always admitted."""
    from collections import deque
    from types import SimpleNamespace

    from atomx_b200.serve import SlaterServer

    def take(srv, q, used, busy):
        group, fp = SlaterServer._take_group(srv, q, used, busy)
        assert fp == sum(r.footprint for r in group)
        return group

    srv = SimpleNamespace(max_group=3, group_bytes=100, hbm_budget=1000)
    q = deque(_req(i, 10) for i in range(5))
    assert [r.rid for r in take(srv, q, 0, False)] == [0, 1, 2] and [r.rid for r in q] == [3, 4]
    q = deque([_req(0, 60), _req(1, 30), _req(2, 20), _req(3, 5)])
    assert [r.rid for r in take(srv, q, 0, False)] == [0, 1]          # 60 + 30 + 20 > group_bytes
    q = deque([_req(0, 400), _req(1, 10)])
    assert take(srv, q, 700, True) == [] and len(q) == 2               # budget full while busy
    assert [r.rid for r in take(srv, q, 700, False)] == [0]            # an idle device takes the head
    q = deque([_req(0, 10), _req(1, 500, streamed=True), _req(2, 10)])
    assert [r.rid for r in take(srv, q, 0, False)] == [0]
    assert [r.rid for r in take(srv, q, 0, False)] == [1]              # a streamed request runs alone
    assert [r.rid for r in take(srv, q, 0, False)] == [2]


def test_serving_group_rows_take_the_widest_row():
    """In a group every ion's rows are padded to the group's widest row, and
    the group's footprint says so."""
    from atomx_b200.serve import _group_footprint
    a, b = _req(0, 0), _req(1, 0)
    a.state["parts"], b.state["parts"] = (100, 10, 256, 30), (50, 20, 1024, 30)
    a.footprint, b.footprint = 100 + 10 * 256 * 30, 50 + 20 * 1024 * 30
    assert _group_footprint([a]) == a.footprint
    assert _group_footprint([a, b]) == 150 + 30 * 1024 * 30 > a.footprint + b.footprint


def test_plan_is_cached_read_only_and_ordered():
    from atomx_b200 import plan as PL
    from atomx_b200 import workloads as W
    kappa = W.build_ion(W.ytterbium_scaleup()).kappa
    p = PL.make_plan(kappa, 12)
    assert PL.make_plan(np.array(kappa), 12) is p and PL.make_plan(kappa, 11) is not p
    for a in (p.pairs, p.row_pair, p.row_k, p.pair_block):
        assert not a.flags.writeable
    # pairs: block by block, a-major; a <= c inside a shell block
    for bi, (ka, kc, s0, s1) in enumerate(p.blocks):
        blk = p.pairs[s0:s1]
        assert np.all(p.pair_block[s0:s1] == bi) and np.all(kappa[blk[:, 0]] == ka) and np.all(kappa[blk[:, 1]] == kc)
        order = blk[:, 0] * len(kappa) + blk[:, 1]
        assert np.all(np.diff(order) > 0)
        if ka == kc:
            assert np.all(blk[:, 0] <= blk[:, 1])
    # rows: grouped by k in increasing order, each group the pairs of that k
    for k in p.ks:
        o, n = p.k_row_offset[k], p.n_of_k(k)
        assert np.array_equal(p.row_pair[o:o + n], p.pairs_of_k[k]) and np.all(p.row_k[o:o + n] == k)
    assert p.row_pair.shape[0] == sum(p.n_of_k(k) for k in p.ks) == p.n_rows


def test_packed_host_tables_expand_symmetric():
    """HostPackedTables (the host format of slater_rk_tables(host=True,
    packed=True)): the packed upper triangle of every multipole table expands
    to the symmetric table, and entry() reads either ordering."""
    import numpy as np
    import torch

    from atomx_b200.plan import make_plan
    from atomx_b200.tables import HostPackedTables, packed_offsets
    plan = make_plan(np.array([-1, -1, 1, -2, -2, 2]), 3)
    offs = packed_offsets(plan)
    rng = np.random.default_rng(3)
    full = {}
    vals = np.zeros(plan.unique_entries)
    for k in plan.ks:
        n = plan.n_of_k(k)
        a = rng.normal(size=(n, n))
        full[k] = a + a.T
        vals[offs[k]:offs[k] + n * (n + 1) // 2] = full[k][np.triu_indices(n)]
    last = plan.ks[-1]
    assert offs[last] + plan.n_of_k(last) * (plan.n_of_k(last) + 1) // 2 == plan.unique_entries
    t = HostPackedTables(plan=plan, ks=plan.ks, values=torch.from_numpy(vals), offsets=offs, precision="fp64")
    for k in plan.ks:
        assert np.array_equal(t.table(k), full[k])
    k = plan.ks[1]
    pr = plan.pairs[plan.pairs_of_k[k]]
    i, j = 0, len(pr) - 1
    assert t.entry(k, tuple(pr[i]), tuple(pr[j])) == full[k][i, j] == t.entry(k, tuple(pr[j]), tuple(pr[i]))
    assert t.ordered_entries == plan.ordered_entries and t.unique_entries == plan.unique_entries
