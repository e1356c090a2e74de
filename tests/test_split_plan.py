"""CPU checks of the split engine's planning: the packed factor tables, the
factored identity R = X.X - Z.Z + left.right against the oracle, the CRT
constants, and the fixed-point error model."""
import numpy as np
import pytest

from oracle import oracle
from split_emulation import crt_value, transform_rows, unpack_table


def _ion_rows(name, n_pairs=120, seed=0):
    from atomx_b200 import plan as PL
    from atomx_b200 import workloads as W
    spec = getattr(W, name)()
    ion = W.build_ion(spec)
    bd = ion.bsp
    Pg = np.array([oracle.eval_P(c, bd).ravel() for c in ion.P])
    Qg = np.array([oracle.eval_Q(c, bd).ravel() for c in ion.Q])
    plan = PL.make_plan(ion.kappa, spec.k_max)
    return spec, ion, bd, Pg, Qg, plan


@pytest.mark.parametrize("name,ks", [("neon_small", [0, 1, 2]), ("ytterbium_scaleup", [0, 5, 12])])
def test_factored_identity_matches_oracle(name, ks):
    from atomx_b200.split import factors_for_grid
    from atomx_b200.split_plan import concat_tables
    spec, ion, bd, Pg, Qg, plan = _ion_rows(name)
    gr, grw = bd["gr"], bd["grw"]
    nv, ng = gr.shape
    facs = factors_for_grid(gr.ravel(), ng, ks)
    flat, offs = concat_tables([facs[k] for k in ks])
    rng = np.random.default_rng(1)
    for i, k in enumerate(ks):
        F = unpack_table(flat, offs[i], nv, ng)
        pk = plan.pairs_of_k[k]
        sel = pk[rng.choice(pk.shape[0], size=min(60, pk.shape[0]), replace=False)]
        rho = np.array([Pg[a] * Pg[c] + Qg[a] * Qg[c] for a, c in plan.pairs[sel]])
        g = rho * grw.reshape(1, -1)
        y = oracle.yk_rows(rho, k, gr, grw, nv, ng)
        ref = g @ y.T
        X, Z, left, right = transform_rows(g, F, nv, ng)
        got = X @ X.T - Z @ Z.T + left @ right.T
        d = np.abs(np.diag(ref))
        err = np.abs(got - ref) / np.sqrt(np.outer(d, d))
        assert err.max() < 1e-13, (name, k, err.max())


@pytest.mark.parametrize("index,ks", [(19, [4, 8]), (16, [4]), (34, [6])])
def test_factored_identity_on_wide_origin_cells(index, ks):
    """Ions of the uneven batch whose first body node sits near 1e-5 with cell
    ratios near 60: the core-body coupling is kept as two FP64 columns, so the
    identity holds to rounding (folding it into X as ell * (v_0.g_0), with
    |ell|^2 ~ r_b^-(2k+1), missed by 2e-3 here even in FP64)."""
    from atomx_b200 import plan as PL
    from atomx_b200 import workloads as W
    from atomx_b200.split import factors_for_grid
    spec = W.uneven_batch()[index]
    ion = W.build_ion(spec)
    bd = ion.bsp
    gr, grw = bd["gr"], bd["grw"]
    nv, ng = gr.shape
    Pg = np.array([oracle.eval_P(c, bd).ravel() for c in ion.P])
    Qg = np.array([oracle.eval_Q(c, bd).ravel() for c in ion.Q])
    plan = PL.make_plan(ion.kappa, spec.k_max)
    rng = np.random.default_rng(index)
    for k in ks:
        F = unpack_table(factors_for_grid(gr.ravel(), ng, [k])[k], 0, nv, ng)
        pk = plan.pairs_of_k[k]
        sel = pk[rng.choice(pk.shape[0], size=min(200, pk.shape[0]), replace=False)]
        rho = np.array([Pg[a] * Pg[c] + Qg[a] * Qg[c] for a, c in plan.pairs[sel]])
        g = rho * grw.reshape(1, -1)
        ref = g @ oracle.yk_rows(rho, k, gr, grw, nv, ng).T
        X, Z, left, right = transform_rows(g, F, nv, ng)
        got = X @ X.T - Z @ Z.T + left @ right.T
        d = np.abs(np.diag(ref))
        assert (np.abs(got - ref) / np.sqrt(np.outer(d, d))).max() < 1e-13, (index, k)
        # the two scaled moments stay within |g|_1 / sqrt(r_b)
        bound = np.abs(g).sum(axis=1) / np.sqrt(gr[1, 0])
        assert np.all(np.abs(left[:, ng:]).max(axis=1) <= bound * (1 + 1e-12))


def test_crt_constants_reconstruct_integers():
    from atomx_b200.split_plan import crt_constants, moduli_needed
    for bits, kdim in ((36, 896), (36, 2176), (40, 1024)):
        nm = moduli_needed(bits, kdim)
        ms, fh, fl, M, pinv = crt_constants(nm)
        assert M > 2 * kdim * 2.0 ** (2 * bits)
        rng = np.random.default_rng(bits)
        bound = kdim * 2 ** (2 * bits)
        xs = [int(v) for v in rng.integers(-2**62, 2**62, size=200)] + [bound, -bound, 0, 1, -1]
        xs = [x % (2 * bound) - bound for x in xs]
        for x in xs:
            res = [np.array([((x + int(m) // 2) % int(m)) - int(m) // 2]) for m in ms]  # any representative
            got = float(crt_value(res, ms, fh, fl, M, pinv)[0])
            assert abs(got - float(x)) <= 2.0 ** -50 * abs(float(x)) + 8.0, (bits, x, got)
        # f_hi exactness: multiples of 2^-34
        assert np.all(fh * 2.0 ** 34 == np.rint(fh * 2.0 ** 34))


def test_fixed_point_split_error_model():
    """36-bit rows: Schwarz-relative error ~ 2^-36 on the Z=70 ion."""
    from atomx_b200.split import factors_for_grid
    spec, ion, bd, Pg, Qg, plan = _ion_rows("ytterbium_scaleup")
    gr, grw = bd["gr"], bd["grw"]
    nv, ng = gr.shape
    for k in (0, 12):
        F = unpack_table(factors_for_grid(gr.ravel(), ng, [k])[k], 0, nv, ng)
        pk = plan.pairs_of_k[k]
        sel = pk[np.random.default_rng(k).choice(pk.shape[0], size=min(200, pk.shape[0]), replace=False)]
        rho = np.array([Pg[a] * Pg[c] + Qg[a] * Qg[c] for a, c in plan.pairs[sel]])
        g = rho * grw.reshape(1, -1)
        X, Z, left, right = transform_rows(g, F, nv, ng)
        XZ = np.concatenate([X, Z], axis=1)
        e = np.frexp(np.abs(XZ).max(axis=1))[1]
        s = np.ldexp(1.0, 36 - e)[:, None]
        q = np.rint(XZ * s) / s
        qm = q.copy()
        qm[:, X.shape[1]:] *= -1
        got = q @ qm.T + left @ right.T
        ref = XZ @ np.concatenate([X, -Z], axis=1).T + left @ right.T
        d = np.abs(np.diag(ref))
        err = np.abs(got - ref) / np.sqrt(np.outer(d, d))
        assert err.max() < 5e-11, (k, err.max())


@pytest.mark.parametrize("name,ks", [("neon_small", [0, 1, 2]), ("ytterbium_scaleup", [0, 3, 12]),
                                     ("xenon_ci_table", [0, 16])])
def test_native_factor_equals_numpy_factor(name, ks):
    """The native factorisation (Jacobi eigensolver) and the numpy one give the
    same packed table; Z columns may differ in sign only (z z^T is the same)."""
    from atomx_b200.split_plan import green_factor, green_factor_packed, pack_factors
    spec, ion, bd, Pg, Qg, plan = _ion_rows(name)
    nv, ng = bd["gr"].shape
    r = bd["gr"].ravel()
    for k in ks:
        a = unpack_table(green_factor_packed(r, ng, k), 0, nv, ng)
        ref_flat, _ = pack_factors([green_factor(r, ng, k)])
        b = unpack_table(ref_flat, 0, nv, ng)
        assert a["sx"] == pytest.approx(b["sx"], rel=1e-14)
        for key in ("u", "Lb", "C", "v0", "G00"):
            scale = np.abs(b[key]).max() + 1e-300
            assert np.abs(a[key] - b[key]).max() <= 1e-11 * scale, (name, k, key)
        np.testing.assert_array_equal(a["zcell"], b["zcell"])
        for m in np.unique(b["zcell"]):
            za, zb = a["zvec"][a["zcell"] == m], b["zvec"][b["zcell"] == m]
            pa, pb = za.T @ za, zb.T @ zb
            assert np.abs(pa - pb).max() <= 1e-10 * (np.abs(pb).max() + 1e-300), (name, k, m)
