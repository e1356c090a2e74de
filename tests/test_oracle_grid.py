"""The arbitrary-grid trapezoid Y^k oracle (oracle/rk_oracle.c, oracle.py)
against golden vectors from atomx's own numerics/quadrature.py
(tests/golden/grid_quadrature.npz, made by tests/golden/make_golden.py).

The oracle restates the serial scans operation by operation, so values must
be identical to the reference's, bit for bit; the one exception is noted in
test_grid_slater_rk_bitwise."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(GOLDEN, "grid_quadrature.npz"))


def test_yk_on_grid_wide_range_bitwise(g):
    for i, k in enumerate(g["a_ranks"]):
        np.testing.assert_array_equal(oracle.yk_on_grid(g["a_rho"], g["a_r"], int(k)), g["a_yk"][i])
        np.testing.assert_array_equal(oracle.yk_on_grid(g["a_rho"], g["a_r"], int(k), i_cut=97), g["a_yk_cut"][i])


def test_grid_slater_rk_bitwise(g):
    r = g["a_r"]
    ones, zeros = np.ones_like(r), np.zeros_like(r)
    for i, k in enumerate(g["a_ranks"]):
        got = oracle.grid_slater_rk(g["a_other"], zeros, g["a_rho"], zeros, ones, zeros, ones, zeros, r, int(k))
        assert got == g["a_slater"][i]
    # With nonzero small components the reference's scalar kernel (one Numba
    # function with the Y^k scan inlined) rounds a few multiply-adds as fused
    # operations; the batched path matches bit for bit (below), this one to
    # a few units in the last place.
    P, Q, rf = g["c_P"], g["c_Q"], g["c_r"]
    for i, k in enumerate((0, 1, 4)):
        got = oracle.grid_slater_rk(P[0], Q[0], P[1], Q[1], P[2], Q[2], P[3], Q[3], rf, k)
        assert got == pytest.approx(g["c_slater"][i], rel=1e-14, abs=0.0)


def test_pair_dot_batch_bitwise(g):
    for cut in (0, 41, 80):
        got = oracle.yk_pair_dot_batch_on_grid(g["b_pa"], g["b_qa"], g["b_pb"], g["b_qb"], g["b_a"], g["b_b"],
                                               g["b_k"], g["b_ok"], g[f"b_outer{cut}"], g["b_ptr"], g["b_cons"],
                                               g["b_r"], i_cut=cut)
        np.testing.assert_array_equal(got, g[f"b_val{cut}"])
    got = oracle.yk_pair_dot_batch_on_grid(g["c_P"], g["c_Q"], g["c_P"], g["c_Q"], g["c_a"], g["c_b"], g["c_k"],
                                           g["c_ok"], g["c_w"], g["c_ptr"], g["c_cons"], g["c_r"],
                                           i_cut=int(g["c_cut"]))
    np.testing.assert_array_equal(got, g["c_val"])


def test_endpoint_rules_bitwise(g):
    r4 = np.array([0.1, 0.4, 1.0, 2.0])
    a4, b4, z4 = np.array([1.0, 2.0, 0.0, 0.0]), np.ones(4), np.zeros(4)
    assert oracle.grid_slater_rk(a4, z4, b4, z4, b4, z4, b4, z4, r4, 0) == float(g["d_cut"])
    r3 = np.array([1e-7, 1.0, 1e20])
    a3, b3, z3 = np.array([1.0, 1e-20, 1e-20]), np.ones(3), np.zeros(3)
    assert oracle.grid_slater_rk(a3, z3, b3, z3, b3, z3, b3, z3, r3, 0) == float(g["d_tail"])


def test_tables_reject_invalid_input():
    with pytest.raises(ValueError):
        oracle.coulomb_tables(np.array([1.0, 0.5]), 2)
    with pytest.raises(ValueError):
        oracle.coulomb_tables(np.array([0.1, 1.0]), -1)
    with pytest.raises(ValueError):
        oracle.coulomb_tables(np.array([0.1, 1.0]), 1.5)
