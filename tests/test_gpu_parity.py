"""Device parity: every drop-in entry point and the plain FP64 table engine
against the oracle and the reference's own golden vectors.

Tolerances:
* Y^k rows: |Y - Y_ref| <= 1e-13 max|Y_ref| per row (the device scan only
  re-associates the cross-cell base sums; measured ~1e-16).
* R^k entries: Schwarz-relative error |R - R_ref| / sqrt(|R_acac R_bdbd|)
  <= 1e-13, and plain relative <= 1e-12 where |R_ref| >= 1e-3 of that scale
  and <= 1e-13 where |R_ref| >= 5e-2 of it (the floored-relative metric over
  the most cancelling entries is in test_gpu_accuracy.py).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="module")
def neon():
    g = _load("neon_small.npz")
    from atomx_b200 import basis
    bd = basis.prepare_bspline_data(g["t"], 40, 7, n_gauss=7, kinetic_balance=True)
    return g, bd


def test_library_loads_and_device_supported():
    from atomx_b200 import _native
    L = _native.require_device()
    assert b"sm_100a" in L.rkb_version()


def test_compute_yk_neon_rows(neon):
    from atomx_b200.yk import compute_yk, compute_yk_rows
    g, bd = neon
    gr, grw = g["gr"], g["grw"]
    nv, ng = gr.shape
    rho = np.array([g["Pg"][a] * g["Pg"][c] + g["Qg"][a] * g["Qg"][c] for a, c in g["pairs"]])
    ref = g["yk_rows"]
    rows = compute_yk_rows(rho[g["row_pair"]], g["row_k"], gr, grw)
    err = np.max(np.abs(rows - ref), axis=1) / np.max(np.abs(ref), axis=1)
    assert err.max() <= 1e-13, err.max()
    for q in range(3):
        one = compute_yk(rho[g["row_pair"][q]].reshape(nv, ng), gr, grw, nv, ng, int(g["row_k"][q]))
        assert one.shape == (nv, ng)
        assert np.max(np.abs(one.ravel() - ref[q])) <= 1e-13 * np.max(np.abs(ref[q]))


def _oracle_values(ion):
    bd = ion.bsp
    Pg = np.array([oracle.eval_P(c, bd).ravel() for c in ion.P])
    Qg = np.array([oracle.eval_Q(c, bd).ravel() for c in ion.Q])
    return Pg, Qg


@pytest.mark.parametrize("name", ["ytterbium_scaleup", "xenon_ci_table"])
def test_yk_rows_large_ions(name):
    """Y^k of the reference's own stored densities against its rows."""
    from atomx_b200 import basis
    from atomx_b200 import workloads as W
    from atomx_b200.yk import compute_yk_rows
    g = _load(f"{name}.npz")
    spec = getattr(W, name)()
    t = basis.make_exponential_knots(spec.ns, spec.ks, spec.r_min, spec.r_max)
    bd = basis.prepare_bspline_data(t, spec.ns, spec.ks, n_gauss=spec.n_gauss, kinetic_balance=True)
    got = compute_yk_rows(g["row_rho"], g["row_k"], bd["gr"], bd["grw"])
    ref = g["yk_rows"]
    err = np.max(np.abs(got - ref), axis=1) / np.max(np.abs(ref), axis=1)
    assert err.max() <= 1e-13, err.max()


def test_yk_high_k_and_odd_ng():
    """k up to 16 and every ng the configs and reference tests use."""
    from atomx_b200 import basis
    from atomx_b200.yk import compute_yk_rows
    rng = np.random.default_rng(3)
    for ng in (2, 5, 7, 8, 9, 11, 14, 17, 21):
        t = basis.make_exponential_knots(60, 9, 1e-6, 60.0)
        gr, grw = basis.setup_gauss_points(t, 60, 9, ng)
        nv = gr.shape[0]
        rho = rng.standard_normal((4, nv * ng)) * np.exp(-gr.ravel())[None, :]
        for k in (0, 3, 16):
            ref = oracle.yk_rows(rho, k, gr, grw, nv, ng)
            got = compute_yk_rows(rho, k, gr, grw)
            err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
            assert err <= 1e-13, (ng, k, err)


def test_complex_density_is_linear():
    from atomx_b200 import basis
    from atomx_b200.yk import compute_yk
    t = basis.make_exponential_knots(40, 7, 1e-5, 40.0)
    gr, grw = basis.setup_gauss_points(t, 40, 7, 7)
    nv, ng = gr.shape
    rng = np.random.default_rng(0)
    re, im = rng.standard_normal((2, nv, ng)) * np.exp(-gr)
    got = compute_yk(re + 1j * im, gr, grw, nv, ng, 2)
    ref = oracle.yk_row(re, gr, grw, nv, ng, 2) + 1j * oracle.yk_row(im, gr, grw, nv, ng, 2)
    assert np.max(np.abs(got.ravel() - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_device_tensor_inputs_stay_on_device():
    from atomx_b200 import basis
    from atomx_b200.yk import compute_yk
    t = basis.make_exponential_knots(40, 7, 1e-5, 40.0)
    gr, grw = basis.setup_gauss_points(t, 40, 7, 7)
    nv, ng = gr.shape
    rho = torch.exp(-torch.as_tensor(gr, device="cuda"))
    y = compute_yk(rho, torch.as_tensor(gr, device="cuda"), torch.as_tensor(grw, device="cuda"), nv, ng, 1)
    assert y.is_cuda and y.shape == (nv, ng)
    ref = oracle.yk_row(rho.cpu().numpy(), gr, grw, nv, ng, 1)
    assert np.max(np.abs(y.cpu().numpy().ravel() - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_errors_match_reference_behaviour(neon):
    from atomx_b200.slater import slater_rk, slater_rk_direct
    from atomx_b200.yk import compute_yk
    g, bd = neon
    gr, grw = g["gr"], g["grw"]
    nv, ng = gr.shape
    rho = np.exp(-gr)
    with pytest.raises(ValueError, match="unknown Slater integrator"):
        slater_rk(rho, rho, bd, 1, method="simpson")
    with pytest.raises(ValueError):
        compute_yk(rho, gr, grw, nv, ng, -1)
    with pytest.raises(ValueError):
        slater_rk_direct(rho, rho, gr.ravel(), grw.ravel(), 0)
    with pytest.raises(ValueError):
        slater_rk_direct(rho, rho, gr, grw, 1.5)


def test_slater_poisson_and_direct_neon(neon):
    from atomx_b200.plan import make_plan
    from atomx_b200.slater import slater_rk, slater_rk_poisson
    g, bd = neon
    gr, grw = g["gr"], g["grw"]
    nv, ng = gr.shape
    rho = np.array([g["Pg"][a] * g["Pg"][c] + g["Qg"][a] * g["Qg"][c] for a, c in g["pairs"]])
    plan = make_plan(g["kappa"], 2)
    for k, i, j, val in g["entries"][::4]:
        k, i, j = int(k), int(i), int(j)
        pa, pb = plan.pairs_of_k[k][i], plan.pairs_of_k[k][j]
        got = slater_rk_poisson(rho[pa], rho[pb], gr, grw, nv, ng, k)
        assert got == pytest.approx(val, rel=1e-13, abs=1e-16)
    for pa, pb, k, val in g["direct"]:
        got = slater_rk(rho[int(pa)], rho[int(pb)], bd, int(k), method="direct")
        assert got == pytest.approx(val, rel=1e-12, abs=1e-15)


def test_compute_slater_rk_neon(neon):
    from atomx_b200.slater_yk import compute_slater_fk, compute_slater_gk, compute_slater_rk
    g, bd = neon
    P, Q = g["P"], g["Q"]
    for (a, b, c, d, k), val in zip(g["quads"], g["compute_slater_rk"]):
        got = compute_slater_rk(P[a], Q[a], P[b], Q[b], P[c], Q[c], P[d], Q[d], bd, int(k))
        assert got == pytest.approx(val, rel=1e-13, abs=1e-16)
    fk = compute_slater_fk(P[0], Q[0], P[1], Q[1], bd, 0)
    assert fk == pytest.approx(compute_slater_rk(P[0], Q[0], P[0], Q[0], P[1], Q[1], P[1], Q[1], bd, 0))
    gk = compute_slater_gk(P[0], Q[0], P[2], Q[2], bd, 1)
    assert gk == pytest.approx(compute_slater_rk(P[0], Q[0], P[2], Q[2], P[2], Q[2], P[0], Q[0], bd, 1))


def test_hydrogenic_closed_forms_on_device():
    from atomx_b200.slater import slater_rk_poisson
    h = _load("hydrogenic.npz")
    gr, grw = h["gr"], h["grw"]
    nv, ng = gr.shape
    rho = 4.0 * gr ** 2 * np.exp(-2.0 * gr)
    exact = [5.0 / 8.0, 3.0 / 8.0, 0.260532333438687426013570914996237633812003225]
    for k in range(3):
        got = slater_rk_poisson(rho, rho, gr, grw, nv, ng, k)
        assert got == pytest.approx(exact[k], rel=1e-10)
        assert got == pytest.approx(h["h1s"][k], rel=1e-14)


@pytest.mark.parametrize("name", ["neon_small", "ytterbium_scaleup"])
def test_orbital_values_condition_bound(name):
    """GPU orbital values against the NumPy einsum of the reference.  Near the
    origin a high-kappa spinor is the sum of strongly cancelling B-spline
    terms, so the comparison is held to the summation's condition bound
    |f_gpu - f_ref| <= 8 eps sum_s |c_s B_s(r)| (plus one ulp)."""
    from atomx_b200 import workloads as W
    from atomx_b200.evaluate import eval_orbitals_on_grid
    ion = W.build_ion(getattr(W, name)())
    bd = ion.bsp
    for coeff, bsp, ks, ns in ((ion.P, bd["bsp_p"], bd["ksp"], bd["nsp"]), (ion.Q, bd["bsp_q"], bd["ksq"], bd["nsq"])):
        got = eval_orbitals_on_grid(coeff, bsp, bd["nv"], ks, ns)
        ref = np.array([oracle.eval_orbital_on_grid(c, bsp, bd["nv"], ks, ns).ravel() for c in coeff])
        bound = np.array([oracle.eval_orbital_on_grid(np.abs(c), np.abs(bsp), bd["nv"], ks, ns).ravel()
                          for c in coeff])
        eps = np.finfo(float).eps
        assert np.all(np.abs(got - ref) <= 8 * eps * bound + eps * np.abs(ref) + 1e-300)


def test_orbital_values_neon(neon):
    from atomx_b200.evaluate import eval_P, eval_Q
    g, bd = neon
    for i in range(4):
        np.testing.assert_allclose(eval_P(g["P"][i], bd).ravel(), g["Pg"][i], rtol=0,
                                   atol=1e-14 * np.abs(g["Pg"]).max())
        np.testing.assert_allclose(eval_Q(g["Q"][i], bd).ravel(), g["Qg"][i], rtol=0,
                                   atol=1e-14 * np.abs(g["Qg"]).max())


def _schwarz_check(tab, k, oracle_vals, idx_i, idx_j, gate=1e-13):
    T = tab.table(k).cpu().numpy()
    diag = np.abs(np.diag(T))
    got = T[idx_i, idx_j]
    scale = np.sqrt(diag[idx_i] * diag[idx_j])
    err = np.abs(got - oracle_vals) / scale
    assert err.max() <= gate, (k, err.max())
    # plain relative error: an FP64 error of ~1e-15 of the Schwarz scale is
    # 1e-12 of an entry at 1e-3 of its scale, 2e-14 at 5e-2
    for frac, rel_gate in ((1e-3, 1e-12), (5e-2, 1e-13)):
        big = np.abs(oracle_vals) >= frac * scale
        rel = np.abs(got - oracle_vals)[big] / np.abs(oracle_vals[big])
        assert rel.size == 0 or rel.max() <= rel_gate, (k, frac, rel.max())


def test_fp64_table_neon_every_entry(neon):
    from atomx_b200 import workloads as W
    from atomx_b200.tables import slater_rk_tables
    g, _ = neon
    ion = W.build_ion(W.neon_small())
    tab = slater_rk_tables(ion, precision="fp64")
    for k in tab.ks:
        T = tab.table(k).cpu().numpy()
        ent = g["entries"][g["entries"][:, 0] == k]
        ii, jj, vals = ent[:, 1].astype(int), ent[:, 2].astype(int), ent[:, 3]
        _schwarz_check(tab, k, vals, ii, jj)
        assert np.max(np.abs(T - T.T)) <= 1e-14 * np.max(np.abs(T))


@pytest.mark.parametrize("name", ["ytterbium_scaleup", "xenon_ci_table"])
def test_fp64_table_large_ions_vs_oracle(name):
    """Whole plain tables against the oracle (the reference algorithm, pinned
    by the golden vectors on the CPU) on the same inputs, at seeded sampled
    entries of every multipole."""
    from atomx_b200 import workloads as W
    from atomx_b200.tables import slater_rk_tables_from_values
    from oracle_entries import sampled_oracle_entries
    spec = getattr(W, name)()
    ion = W.build_ion(spec)
    Pg, Qg = _oracle_values(ion)
    tab = slater_rk_tables_from_values(Pg, Qg, ion.kappa, ion.bsp["gr"], ion.bsp["grw"], spec.k_max,
                                       precision="fp64")
    for k, ii, jj, ref in sampled_oracle_entries(ion, Pg, Qg, tab.plan, per_k=48, seed=3):
        _schwarz_check(tab, k, ref, ii, jj)
    # size-independent properties over the whole table
    assert tab.values.numel() == tab.plan.ordered_entries
    assert bool(torch.isfinite(tab.values).all())
    for k in tab.ks:
        T = tab.table(k)
        d = torch.diagonal(T)
        # self-repulsion of a pair density is positive (Coulomb kernel is positive)
        assert bool((d > 0).all()), k


def test_fp64_table_from_coefficients_ytterbium():
    """The coefficient path (GPU orbital values) agrees with the values path
    (NumPy orbital values).  They differ only by the orbital summation's
    rounding, which the cancelling B-spline sums of high-kappa spinors near
    the origin amplify; gate 1e-10 Schwarz-relative."""
    from atomx_b200 import workloads as W
    from atomx_b200.tables import slater_rk_tables, slater_rk_tables_from_values
    ion = W.build_ion(W.ytterbium_scaleup())
    Pg, Qg = _oracle_values(ion)
    a = slater_rk_tables(ion, precision="fp64")
    b = slater_rk_tables_from_values(Pg, Qg, ion.kappa, ion.bsp["gr"], ion.bsp["grw"], 12, precision="fp64")
    for k in a.ks:
        A, B = a.table(k), b.table(k)
        d = torch.sqrt(torch.outer(torch.diagonal(B).abs(), torch.diagonal(B).abs()))
        assert float(((A - B).abs() / d).max()) <= 1e-10, k


def test_pair_density_entry_point_matches_oracle_bitwise(neon):
    """rkb_pair_density (atomx slater_yk.py:193-194, rho = P_aP_c + Q_aQ_c)
    through the C ABI: every pair of the Z=10 table, with strided rows,
    equal to the oracle bit for bit (two products, one add, no fused
    multiply-add on either side)."""
    from atomx_b200 import _native
    L = _native.require_device()
    g, _ = neon
    Pg, Qg, pairs = g["Pg"], g["Qg"], np.ascontiguousarray(g["pairs"], dtype=np.int64)
    n_orb, n = Pg.shape
    ld = n + 5
    P = torch.zeros((n_orb, ld), dtype=torch.float64, device="cuda")
    Q = torch.zeros_like(P)
    P[:, :n] = torch.from_numpy(Pg)
    Q[:, :n] = torch.from_numpy(Qg)
    dp = torch.from_numpy(pairs).cuda()
    rho_ld = n + 3
    rho = torch.full((pairs.shape[0], rho_ld), -7.0, dtype=torch.float64, device="cuda")
    _native.check(L.rkb_pair_density(P.data_ptr(), Q.data_ptr(), ld, dp.data_ptr(), pairs.shape[0], n,
                                     rho.data_ptr(), rho_ld, None), "rkb_pair_density")
    torch.cuda.synchronize()
    got = rho.cpu().numpy()
    ref = np.array([oracle.pair_density(Pg[a], Qg[a], Pg[c], Qg[c]) for a, c in pairs])
    assert np.array_equal(got[:, :n], ref)
    assert np.all(got[:, n:] == -7.0)  # padding columns untouched
    # an empty pair list is a no-op; a leading dimension below n is refused
    _native.check(L.rkb_pair_density(P.data_ptr(), Q.data_ptr(), ld, dp.data_ptr(), 0, n, rho.data_ptr(),
                                     rho_ld, None))
    with pytest.raises(ValueError):
        _native.check(L.rkb_pair_density(P.data_ptr(), Q.data_ptr(), n - 1, dp.data_ptr(), 1, n, rho.data_ptr(),
                                         rho_ld, None))
