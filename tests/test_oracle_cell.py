"""The cell-engine oracle (oracle/cell_oracle.c + oracle/cell.py) against the
golden vectors of atomx's own cell engine (tests/golden/convol.npz, made by
tests/golden/make_golden.py --only convol).

Bit for bit where atomx runs its loops without fastmath (moments, diagonal
cells, banks, the full-bank scalar path, exchange contractions); to a few
ulps of the result's scale where atomx uses fastmath (_convol_case1_t, the
direct density accumulation) or its factored path (ns >= 96).
"""
import numpy as np
import pytest

import cell_fixtures as F
from oracle import cell as C


@pytest.fixture(scope="module")
def gold():
    return F.load()


def _tiny(g):
    return F.basis(g, "tiny")


def test_gauss_legendre_01():
    x, w = C.gl01(9)
    xr, wr = np.polynomial.legendre.leggauss(9)
    assert np.allclose(np.sort(x), 0.5 * (xr + 1), atol=1e-15) and abs(w.sum() - 1.0) < 1e-14


@pytest.mark.parametrize("k", [0, 1, 3])
def test_moments_and_diagonal_cells_bitwise(gold, k):
    bd = _tiny(gold)
    for comp, ks, b in (("p", bd["ksp"], bd["bsp_p"]), ("q", bd["ksq"], bd["bsp_q"])):
        assert np.array_equal(C.moments(b, bd["gr"], bd["grw"], bd["nv"], ks, k), gold[f"tiny_rising_{comp}_{k}"])
        assert np.array_equal(C.moments(b, bd["gr"], bd["grw"], bd["nv"], ks, -(k + 1)),
                              gold[f"tiny_falling_{comp}_{k}"])
    assert np.array_equal(C.triang(bd["bsp_p"], bd["bsp_p"], bd["gr"], bd["grw"], bd["tp"], bd["tp"], bd["nv"],
                                   bd["ksp"], bd["ksp"], True, k), gold[f"tiny_diag_pppp_{k}"])
    assert np.array_equal(C.triang(bd["bsp_p"], bd["bsp_q"], bd["gr"], bd["grw"], bd["tp"], bd["t"], bd["nv"],
                                   bd["ksp"], bd["ksq"], False, k), gold[f"tiny_diag_pqpq_{k}"])


@pytest.mark.parametrize("k", [0, 1, 3])
@pytest.mark.parametrize("itype", C.ITYPES)
def test_banks_bitwise(gold, k, itype):
    bd = _tiny(gold)
    rkb, ns, ks = C.get_rkb(bd, k, itype)
    ref = gold[f"tiny_rkb_{itype}_{k}"]
    assert rkb.shape == ref.shape and ns == bd["ns"]
    assert np.array_equal(rkb, ref)


class _Ion:
    def __init__(self, g, name):
        self.bsp = F.basis(g, name)
        od = F.orbitals(g, name)
        n = max(od) + 1
        self.P = np.zeros((n, self.bsp["ns"]))
        self.Q = np.zeros((n, self.bsp["ns"]))
        for i, (p, q) in od.items():
            self.P[i], self.Q[i] = p, q


def _neon(g):
    return _Ion(g, "neon")


def test_scalar_cell_integrals_neon_bitwise(gold):
    ion = _neon(gold)
    bd, banks = ion.bsp, C.Banks(ion.bsp)
    keys, ref = gold["neon_keys"], gold["neon_cell"]
    got = np.array([C.slater_rk_cell(ion.P[a], ion.Q[a], ion.P[b], ion.Q[b], ion.P[c], ion.Q[c], ion.P[d], ion.Q[d],
                                     bd, int(k), banks) for a, b, c, d, k in keys])
    assert np.array_equal(got, ref)
    # atomx's batched kernel sums in another order: equal to ~1e-14
    assert np.max(np.abs(gold["neon_batch"] - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_bilinear_and_table_neon(gold):
    ion = _neon(gold)
    bd, banks = ion.bsp, C.Banks(ion.bsp)
    M = C.build_slater_rk_bilinear(ion.P[0], ion.Q[0], ion.P[1], ion.Q[1], bd, 1, banks)
    for name, m in zip(("PP", "QQ", "PQ", "QP"), M):
        assert np.array_equal(m, gold[f"neon_bilinear_{name}"]), name
    tab = C.slater_rk_table(M, ion.P.T, ion.Q.T, ion.P.T, ion.Q.T)
    assert np.allclose(tab, gold["neon_bilinear_table"], rtol=0, atol=1e-15 * np.abs(tab).max())


def test_direct_and_exchange_matrices_neon(gold):
    ion = _neon(gold)
    bd, banks = ion.bsp, C.Banks(ion.bsp)
    J = C.direct_potential_cell(ion.P[1], ion.Q[1], bd, 1, banks)
    for name, m in zip(("PP", "QQ"), J):
        ref = gold[f"neon_direct_{name}"]
        assert np.max(np.abs(m - ref)) <= 1e-14 * np.abs(ref).max(), name  # case 1 is fastmath in atomx
    K = C.exchange_matrix_cell(ion.P[1], ion.Q[1], ion.P[2], ion.Q[2], bd, 1, banks)
    for name, m in zip(("PP", "QQ", "PQ", "QP"), K):
        assert np.array_equal(m, gold[f"neon_exchange_{name}"]), name


def test_dbsr_fock_blocks_neon(gold):
    ion = _neon(gold)
    bd, banks = ion.bsp, C.Banks(ion.bsp)
    n = ion.P.shape[0]
    ad, ax, norms = gold["neon_hf_angular_direct"], gold["neon_hf_angular_exchange"], gold["neon_hf_norms"]
    ref = gold["neon_hf"]
    for target in range(n):
        for s, skip in enumerate((False, True)):
            got = np.stack(C.hf_matrix_dbsr(target, ion.P, ion.Q, ad, ax, range(3), norms[target], bd, banks, skip))
            want = ref[2 * target + s]
            assert np.max(np.abs(got - want)) <= 1e-14 * np.abs(want).max(), (target, skip)


def test_scalar_cell_integrals_ytterbium(gold):
    """ns = 120: atomx's scalar path is the factored one; the oracle's full
    bank gives the same integrals to ~1e-12 of the largest, and atomx's own
    batched kernel (full bank) agrees with the oracle more closely."""
    ion = _Ion(gold, "yb")
    bd, banks = ion.bsp, C.Banks(ion.bsp)
    keys = gold["yb_keys"][:24]
    got = np.array([C.slater_rk_cell(ion.P[a], ion.Q[a], ion.P[b], ion.Q[b], ion.P[c], ion.Q[c], ion.P[d], ion.Q[d],
                                     bd, int(k), banks) for a, b, c, d, k in keys])
    scale = np.abs(gold["yb_cell"]).max()
    assert np.max(np.abs(got - gold["yb_cell"][:24])) <= 1e-11 * scale
    assert np.max(np.abs(got - gold["yb_batch"][:24])) <= 1e-13 * scale
