"""Device cell (bank) engine against atomx's own cell engine (golden vectors
in tests/golden/convol.npz) and against the oracle (the cell algorithm
restated in C) on the same inputs.

Gates:
* banks, moments and diagonal cells: bit for bit (atomx's operation order,
  every product and sum rounded separately);
* exchange matrices (atomx's _convol_case4_t order): bit for bit;
* bilinear matrices (_rkb_bilinear order): bit for bit;
* cell integrals, tables, direct matrices and Fock blocks, which the device
  contracts as FP64 GEMMs in another summation order: 1e-13 of the
  largest magnitude in the set (atomx's own batched and scalar kernels differ
  by 4.5e-14 relative, tests/test_slater_batch_parity.py:4-8), and 1e-11 on
  the Z=70 basis where atomx's scalar path is its factored one (which differs
  from the full bank by ~2e-12).
"""
import numpy as np
import pytest

import cell_fixtures as F
from oracle import cell as OC

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def gold():
    return F.load()


def _tiny(g):
    return F.basis(g, "tiny")


class _Ion:
    """The stored basis and spinors of one fixture ion (as atomx saw them)."""

    def __init__(self, g, name):
        self.bsp = F.basis(g, name)
        od = F.orbitals(g, name)
        n = max(od) + 1
        self.P = np.zeros((n, self.bsp["ns"]))
        self.Q = np.zeros((n, self.bsp["ns"]))
        for i, (p, q) in od.items():
            self.P[i], self.Q[i] = p, q
        self.od = od


def _ion(name):
    from atomx_b200 import workloads as W
    return W.build_ion(getattr(W, name)())


def _close(got, ref, tol):
    got, ref = np.asarray(got), np.asarray(ref)
    scale = np.abs(ref).max()
    err = np.abs(got - ref).max() / scale
    assert err <= tol, err
    return err


@pytest.mark.parametrize("k", [0, 1, 3])
def test_device_banks_bitwise_tiny(gold, k):
    from atomx_b200.convol import ITYPES, ConvolCache
    bd = _tiny(gold)
    cache = ConvolCache(bd)
    cache.release_shared_banks()
    for itype in ITYPES:
        rkb, ns, ks = cache.get_rkb(k, itype)
        ref = gold[f"tiny_rkb_{itype}_{k}"]
        assert rkb.shape == ref.shape and ns == bd["ns"]
        assert np.array_equal(rkb, ref), itype
        rkbT, _, _ = cache.get_rkb_t(k, itype)
        assert np.array_equal(rkbT, ref.transpose(2, 3, 0, 1))
    b = cache.bank(k)
    for comp in ("p", "q"):
        assert np.array_equal(b.moments[comp, "rising"].cpu().numpy(), gold[f"tiny_rising_{comp}_{k}"])
        assert np.array_equal(b.moments[comp, "falling"].cpu().numpy(), gold[f"tiny_falling_{comp}_{k}"])


@pytest.mark.parametrize("name,ks_", [("neon", (0, 1, 2)), ("yb", (0, 5, 12))])
def test_device_banks_bitwise_vs_oracle(gold, name, ks_):
    """Whole banks of the Z=10 (ns=40) and Z=70 (ns=120) bases, every
    component pair, against the oracle restatement of atomx's builder."""
    from atomx_b200.convol import ITYPES, ConvolCache
    bd = F.basis(gold, name)
    cache = ConvolCache(bd)
    for k in ks_:
        for itype in ITYPES:
            got, _, _ = cache.get_rkb(k, itype)
            ref, _, _ = OC.get_rkb(bd, k, itype)
            assert np.array_equal(got, ref), (k, itype)


def test_cell_integrals_neon(gold):
    from atomx_b200 import convol as C
    ion = _Ion(gold, "neon")
    bd, od = ion.bsp, ion.od
    keys = [tuple(int(x) for x in kk) for kk in gold["neon_keys"]]
    got = np.array(C.compute_slater_rk_cell_batch(od, keys, bd))
    _close(got, gold["neon_cell"], 1e-13)
    _close(got, gold["neon_batch"], 1e-13)
    a, b, c, d, k = keys[7]
    one = C.compute_slater_rk_cell(*od[a], *od[b], *od[c], *od[d], bd, k)
    assert abs(one - gold["neon_cell"][7]) <= 1e-13 * np.abs(gold["neon_cell"]).max()
    f0 = C.compute_slater_fk_cell(*od[0], *od[1], bd, 0)
    g0 = C.compute_slater_gk_cell(*od[0], *od[1], bd, 0)
    banks = OC.Banks(bd)
    assert f0 == pytest.approx(OC.slater_rk_cell(*od[0], *od[0], *od[1], *od[1], bd, 0, banks), rel=1e-13)
    assert g0 == pytest.approx(OC.slater_rk_cell(*od[0], *od[1], *od[1], *od[0], bd, 0, banks), rel=1e-13)


def test_cell_integrals_ytterbium(gold):
    from atomx_b200 import convol as C
    ion = _Ion(gold, "yb")
    od = ion.od
    keys = [tuple(int(x) for x in kk) for kk in gold["yb_keys"]]
    got = np.array(C.compute_slater_rk_cell_batch(od, keys, ion.bsp))
    _close(got, gold["yb_batch"], 1e-13)   # atomx's full-bank batch kernel
    _close(got, gold["yb_cell"], 1e-11)    # atomx's factored scalar path


def test_bilinear_and_table_neon(gold):
    from atomx_b200 import convol as C
    ion = _Ion(gold, "neon")
    M = C.build_slater_rk_bilinear(ion.P[0], ion.Q[0], ion.P[1], ion.Q[1], ion.bsp, 1)
    for name, m in zip(("PP", "QQ", "PQ", "QP"), M):
        assert np.array_equal(m, gold[f"neon_bilinear_{name}"]), name
    tab = C.compute_slater_rk_table(M, ion.P.T, ion.Q.T, ion.P.T, ion.Q.T)
    _close(tab, gold["neon_bilinear_table"], 1e-14)
    v = C.eval_slater_rk_bilinear(M, ion.P[2], ion.Q[2], ion.P[3], ion.Q[3])
    assert v == pytest.approx(gold["neon_bilinear_table"][2, 3], rel=1e-13)


def test_bilinear_table_ytterbium(gold):
    from atomx_b200 import convol as C
    ion = _Ion(gold, "yb")
    M = C.build_slater_rk_bilinear(ion.P[0], ion.Q[0], ion.P[9], ion.Q[9], ion.bsp, 2)
    cols = gold["yb_table_cols"]
    tab = C.compute_slater_rk_table(M, ion.P[cols].T, ion.Q[cols].T, ion.P[cols].T, ion.Q[cols].T)
    _close(tab, gold["yb_bilinear_table"], 1e-13)


def test_direct_and_exchange_matrices_neon(gold):
    from atomx_b200 import convol as C
    ion = _Ion(gold, "neon")
    bd = ion.bsp
    J = C.compute_direct_potential_cell(ion.P[1], ion.Q[1], bd, 1)
    for name, m in zip(("PP", "QQ"), J):
        _close(m, gold[f"neon_direct_{name}"], 1e-13)
    K = C.compute_exchange_matrix_cell(ion.P[1], ion.Q[1], ion.P[2], ion.Q[2], bd, 1)
    for name, m in zip(("PP", "QQ", "PQ", "QP"), K):
        assert np.array_equal(m, gold[f"neon_exchange_{name}"]), name
    # the same orbital on both sides: symmetric halves, K_QP = K_PQ^T
    P, Q = ion.P[0], ion.Q[0]
    Kd = C.compute_exchange_matrix_cell(P, Q, P, Q, bd, 2)
    Kr = OC.exchange_matrix_cell(P, Q, P, Q, bd, 2)
    for got, ref in zip(Kd, Kr):
        assert np.array_equal(got, ref)
    assert np.array_equal(Kd[3], Kd[2].T)


@pytest.mark.parametrize("name,tol", [("neon", 1e-13), ("yb", 1e-11)])
def test_direct_exchange_projections(gold, name, tol):
    from atomx_b200 import convol as C
    ion = _Ion(gold, name)
    bd = ion.bsp
    vecs = gold[f"{name}_proj_vecs"]
    orbs = sorted({int(r[1]) for r in gold[f"{name}_direct_proj"]})
    for row_j, row_k in zip(gold[f"{name}_direct_proj"], gold[f"{name}_exchange_proj"]):
        k, o = int(row_j[0]), int(row_j[1])
        slot = orbs.index(o)
        a, b = vecs[2 * slot], vecs[2 * slot + 1]
        J = C.compute_direct_potential_cell(ion.P[o], ion.Q[o], bd, k)
        K = C.compute_exchange_matrix_cell(ion.P[o], ion.Q[o], ion.P[o], ion.Q[o], bd, k)
        gj = np.array([a[0] @ J[0] @ b[0], a[1] @ J[1] @ b[1]])
        gk = np.array([a[0] @ K[0] @ b[0], a[1] @ K[1] @ b[1], a[0] @ K[2] @ b[1], a[1] @ K[3] @ b[0]])
        _close(gj, row_j[2:], tol)
        _close(gk, row_k[2:], tol)


def test_direct_exchange_contract_to_cell_integrals():
    """atomx's own consistency test (tests/test_convol.py:410-437) on the
    device: the direct and exchange blocks of a density c contracted with
    random bra/ket vectors equal the cell integrals R^k(ab, cc) and
    R^k(ac, cb), at 3e-13 relative."""
    from atomx_b200 import basis
    from atomx_b200 import convol as C
    ns, ks = 50, 9
    t = basis.make_exponential_knots(ns, ks, 0.025, 40.0)
    bd = basis.prepare_bspline_data(t, ns, ks, n_gauss=ks)
    rng = np.random.default_rng(713)
    a, b, c = [tuple(rng.normal(size=ns) for _ in range(2)) for _ in range(3)]
    for rank in (0, 1, 2):
        jpp, jqq = C.compute_direct_potential_cell(*c, bd, rank)
        kpp, kqq, kpq, kqp = C.compute_exchange_matrix_cell(*c, *c, bd, rank)
        direct = a[0] @ jpp @ b[0] + a[1] @ jqq @ b[1]
        exchange = a[0] @ kpp @ b[0] + a[1] @ kqq @ b[1] + a[0] @ kpq @ b[1] + a[1] @ kqp @ b[0]
        ej = C.compute_slater_rk_cell(*a, *b, *c, *c, bd, rank)
        ek = C.compute_slater_rk_cell(*a, *c, *c, *b, bd, rank)
        assert direct == pytest.approx(ej, rel=3e-13, abs=1e-11)
        assert exchange == pytest.approx(ek, rel=3e-13, abs=1e-11)
        assert np.array_equal(kpq, kqp.T)


def test_dbsr_fock_blocks_neon(gold):
    from atomx_b200 import convol as C
    ion = _Ion(gold, "neon")
    n = ion.P.shape[0]
    ad, ax, norms = gold["neon_hf_angular_direct"], gold["neon_hf_angular_exchange"], gold["neon_hf_norms"]
    for s, skip in enumerate((False, True)):
        H = C.build_hf_matrices_dbsr(list(range(n)), ion.P, ion.Q, ad, ax, range(3), norms, ion.bsp,
                                     skip_pq_exchange=skip).cpu().numpy()
        for target in range(n):
            _close(H[target], gold["neon_hf"][2 * target + s], 1e-13)
    one = C.build_hf_matrix_dbsr(2, ion.P, ion.Q, ad, ax, range(3), norms[2], ion.bsp)
    _close(np.stack(one), gold["neon_hf"][4], 1e-13)


def test_cell_tables_against_batch_and_poisson():
    """Whole cell tables over every allowed pair of the Z=10 ion: equal to
    the batched integrals, symmetric, and within the known cell-vs-Poisson
    quadrature difference (<= 8e-12 on this basis) of the Poisson engine."""
    from atomx_b200 import convol as C
    from atomx_b200.tables import slater_rk_tables
    ion = _ion("neon_small")
    tab = C.cell_tables(ion.P, ion.Q, ion.kappa, ion.bsp, 2)
    od = {i: (ion.P[i], ion.Q[i]) for i in range(ion.P.shape[0])}
    pois = slater_rk_tables(ion, precision="fp64")
    for k in tab.ks:
        T = tab.table(k).cpu().numpy()
        pr = tab.plan.pairs[tab.plan.pairs_of_k[k]]
        keys = [(a, c, b, d, k) for a, c in pr for b, d in pr]
        ref = np.array(C.compute_slater_rk_cell_batch(od, keys, ion.bsp)).reshape(T.shape)
        _close(T, ref, 1e-13)
        # R^k(ac;bd) = R^k(bd;ac): off-diagonal tiles are mirrored, diagonal
        # tiles compute both orders, which agree to rounding
        _close(T, T.T, 1e-14)
        _close(T, pois.table(k).cpu().numpy(), 1e-10)


def test_pair_potentials_and_radial_evaluator(gold):
    from atomx_b200 import convol as C
    ion = _Ion(gold, "neon")
    bd, od = ion.bsp, ion.od
    ev = C.radial_evaluator(od, bd, pair_potential_cache_size=3)
    # R^k(ac, bd): key ("r", k, a, c, b, d) equals compute_slater_rk_cell(a, c, b, d)
    keys = [("r", int(k), int(a), int(b), int(c), int(d)) for a, b, c, d, k in gold["neon_keys"][:60]]
    got = ev.many(keys)
    _close(got, gold["neon_cell"][:60], 1e-13)
    assert ev(keys[5]) == pytest.approx(gold["neon_cell"][5], rel=1e-12, abs=1e-14)
    info = ev.pair_cache_info()
    assert info["size"] <= 3 and info["misses"] > 0
    # one explicit pair density through the operator (matrix.py:703)
    ns, orders = bd["ns"], (bd["ksp"], bd["ksq"])
    src = (OC.density_sym(ion.P[1], ion.P[2], ns, orders[0]), OC.density_sym(ion.Q[1], ion.Q[2], ns, orders[1]))
    vp, vq = C.bspline_pair_potential(C.ConvolCache(bd), ns, orders, 1, src)
    banks = OC.Banks(bd)
    rp = OC.convol_case1(banks(1, "pppp"), src[0], ns, orders[0], orders[0]) + \
        OC.convol_case1(banks(1, "pqpq"), src[1], ns, orders[0], orders[1])
    rq = OC.convol_case1(banks(1, "qpqp"), src[0], ns, orders[1], orders[0]) + \
        OC.convol_case1(banks(1, "qqqq"), src[1], ns, orders[1], orders[1])
    _close(vp, rp, 1e-13)
    _close(vq, rq, 1e-13)
    with pytest.raises(ValueError):
        C.radial_evaluator(od, bd, pair_potential_cache_size=0)


def test_errors_follow_atomx():
    from atomx_b200 import convol as C
    ion = _ion("neon_small")
    cache = C.ConvolCache(ion.bsp)
    with pytest.raises(ValueError):
        cache.get_rkb(0, "pqqp")
    with pytest.raises(TypeError):
        C.ConvolCache([1, 2, 3])
    bad = ion.P[0].copy()
    bad[3] = np.nan
    with pytest.raises(FloatingPointError):
        C.compute_slater_rk_cell(bad, ion.Q[0], *([ion.P[0], ion.Q[0]] * 3), ion.bsp, 0)
    assert C.compute_slater_rk_cell_batch({}, [], ion.bsp) == []
