"""Arbitrary-grid trapezoid Y^k on the device against the oracle and atomx.

The device scans sum inside each frame in a different order from atomx's
serial loop. So values are compared to the oracle and to the reference's
golden vectors within 1e-13 of the largest |value| of each result. They are
also compared to independent dense Green matrices at the reference's own test
tolerances (rtol 5e-13, atol 2e-14).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = 1e-13


def _close(got, ref, tol=TOL):
    got, ref = np.asarray(got), np.asarray(ref)
    scale = np.abs(ref).max() if ref.size else 1.0
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= tol * max(scale, 1e-300), np.abs(got - ref).max() / scale


def _weights(r):
    out = np.zeros_like(r)
    out[:-1] += 0.5 * np.diff(r)
    out[1:] += 0.5 * np.diff(r)
    return out


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(GOLDEN, "grid_quadrature.npz"))


def test_yk_on_grid_wide_range(g):
    from atomx_b200.quadrature import yk_on_grid
    for i, k in enumerate(g["a_ranks"]):
        _close(yk_on_grid(g["a_rho"], g["a_r"], int(k)), g["a_yk"][i])
        _close(yk_on_grid(g["a_rho"], g["a_r"], int(k), i_cut=97), g["a_yk_cut"][i])


@pytest.mark.parametrize("rank", [0, 1, 12, 32, 64, 128, 256])
def test_dense_green_matrix(rank):
    """The reference's test_scaled_action_and_slater_agree_with_dense_green_matrix."""
    from atomx_b200.quadrature import grid_slater_rk, yk_on_grid, yk_pair_dot_batch_on_grid
    r = np.geomspace(1e-9, 100.0, 193)
    rho = np.sin(3 * np.log(r)) * np.exp(-r / 12)
    other = np.cos(np.log(r)) * np.exp(-r / 9)
    lo, hi = np.minimum(r[:, None], r), np.maximum(r[:, None], r)
    reference = ((lo / hi) ** rank / hi) @ (_weights(r) * rho)
    np.testing.assert_allclose(yk_on_grid(rho, r, rank), reference, atol=2e-14, rtol=5e-13)
    ones, zeros = np.ones_like(r), np.zeros_like(r)
    expected = (other * _weights(r)) @ reference
    assert grid_slater_rk(other, zeros, rho, zeros, ones, zeros, ones, zeros, r, rank) == pytest.approx(
        expected, rel=5e-13, abs=2e-14)
    assert grid_slater_rk(rho, zeros, other, zeros, ones, zeros, ones, zeros, r, rank) == pytest.approx(
        expected, rel=5e-13, abs=2e-14)
    batched = yk_pair_dot_batch_on_grid(rho[None, :], zeros[None, :], ones[None, :], zeros[None, :], np.array([0]),
                                        np.array([0]), np.array([rank]), np.array([True]),
                                        (other * _weights(r))[None, :], np.array([0, 1]), np.array([0]), r)
    assert batched[0] == pytest.approx(expected, rel=5e-13, abs=2e-14)


def test_batch_geometry_and_fine_grid(g):
    from atomx_b200.quadrature import yk_pair_dot_batch_on_grid
    for cut in (0, 41, 80):
        got = yk_pair_dot_batch_on_grid(g["b_pa"], g["b_qa"], g["b_pb"], g["b_qb"], g["b_a"], g["b_b"], g["b_k"],
                                        g["b_ok"], g[f"b_outer{cut}"], g["b_ptr"], g["b_cons"], g["b_r"], i_cut=cut)
        _close(got, g[f"b_val{cut}"])
        # the invalid row's slots stay zero, the empty row has none
        assert np.all(got[2:5] == 0.0)
    got = yk_pair_dot_batch_on_grid(g["c_P"], g["c_Q"], g["c_P"], g["c_Q"], g["c_a"], g["c_b"], g["c_k"], g["c_ok"],
                                    g["c_w"], g["c_ptr"], g["c_cons"], g["c_r"], i_cut=int(g["c_cut"]))
    _close(got, g["c_val"])


def test_grid_slater_rk_fine_grid_and_endpoints(g):
    from atomx_b200.quadrature import grid_slater_rk
    P, Q, rf = g["c_P"], g["c_Q"], g["c_r"]
    for i, k in enumerate((0, 1, 4)):
        assert grid_slater_rk(P[0], Q[0], P[1], Q[1], P[2], Q[2], P[3], Q[3], rf, k) == pytest.approx(
            g["c_slater"][i], rel=1e-13)
    r4 = np.array([0.1, 0.4, 1.0, 2.0])
    a4, b4, z4 = np.array([1.0, 2.0, 0.0, 0.0]), np.ones(4), np.zeros(4)
    assert grid_slater_rk(a4, z4, b4, z4, b4, z4, b4, z4, r4, 0) == pytest.approx(float(g["d_cut"]), rel=3e-14)
    r3 = np.array([1e-7, 1.0, 1e20])
    a3, b3, z3 = np.array([1.0, 1e-20, 1e-20]), np.ones(3), np.zeros(3)
    assert grid_slater_rk(a3, z3, b3, z3, b3, z3, b3, z3, r3, 0) == pytest.approx(float(g["d_tail"]), rel=3e-14)


def test_long_grid_many_rows_against_oracle():
    """120 000 points (many tiles per frame) and ranks that split the grid
    into several frames; 40 rows with up to 3 consumers each."""
    from atomx_b200.quadrature import yk_pair_dot_batch_on_grid
    rng = np.random.default_rng(5)
    r = np.geomspace(1e-4, 60.0, 120_000)
    env = np.exp(-r / 8.0)
    P = rng.normal(size=(5, r.shape[0])) * env
    Q = 0.02 * rng.normal(size=(5, r.shape[0])) * env
    rows = 40
    a, b = rng.integers(0, 5, rows), rng.integers(0, 5, rows)
    ks = rng.integers(0, 40, rows)
    ok = rng.random(rows) > 0.1
    counts = rng.integers(0, 4, rows)
    ptr = np.concatenate([[0], np.cumsum(counts)])
    cons = rng.integers(0, 3, ptr[-1])
    cut = 100_000
    W = rng.normal(size=(3, cut + 1)) * np.exp(-r[:cut + 1] / 10.0)
    got = yk_pair_dot_batch_on_grid(P, Q, P, Q, a, b, ks, ok, W, ptr, cons, r, i_cut=cut)
    ref = oracle.yk_pair_dot_batch_on_grid(P, Q, P, Q, a, b, ks, ok, W, ptr, cons, r, i_cut=cut)
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-13 * np.abs(ref).max())


def test_device_tensors_stay_on_device_and_grid_edits_are_seen():
    from atomx_b200.quadrature import yk_on_grid
    r = np.geomspace(0.1, 10.0, 30)
    rho = np.exp(-r)
    y_dev = yk_on_grid(torch.as_tensor(rho, device="cuda"), r, 3)
    assert isinstance(y_dev, torch.Tensor) and y_dev.is_cuda
    _close(y_dev.cpu().numpy(), oracle.yk_on_grid(rho, r, 3))
    r2 = r * 2  # a different grid must not reuse the first grid's tables
    green = (np.minimum(r2[:, None], r2) / np.maximum(r2[:, None], r2)) ** 3 / np.maximum(r2[:, None], r2)
    np.testing.assert_allclose(yk_on_grid(rho, r2, 3), green @ (_weights(r2) * rho), rtol=5e-14)


def test_errors_match_reference():
    from atomx_b200.quadrature import grid_slater_rk, yk_on_grid
    r = np.geomspace(0.1, 10.0, 30)
    with pytest.raises(ValueError):
        yk_on_grid(np.ones(30), r[::-1], 1)
    with pytest.raises(ValueError):
        yk_on_grid(np.ones(30), r, -1)
    with pytest.raises(ValueError):
        yk_on_grid(np.ones(30), r, 1.5)
    z = np.zeros(30)
    with pytest.raises(ValueError):
        grid_slater_rk(z, z, z, z, z, z, z, z, np.concatenate([[0.0], r[1:]]), 0)
