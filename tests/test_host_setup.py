"""Host-side set-up (knots, grid, B-splines, Dirac spinors, plan) against the
reference's own arrays and the survey's counts."""
import os

import numpy as np
import pytest

from conftest import GOLDEN


def test_neon_basis_bitwise():
    from atomx_b200 import basis
    g = np.load(os.path.join(GOLDEN, "neon_small.npz"))
    t = basis.make_exponential_knots(40, 7, 1e-5, 40.0)
    np.testing.assert_array_equal(t, g["t"])
    bd = basis.prepare_bspline_data(t, 40, 7, n_gauss=7, kinetic_balance=True)
    for key in ("gr", "grw", "bsp_p", "bsp_q"):
        np.testing.assert_array_equal(bd[key], g[key])


def test_neon_spinors_match_reference_eigenvectors():
    from atomx_b200 import workloads as W
    g = np.load(os.path.join(GOLDEN, "neon_small.npz"))
    ion = W.build_ion(W.neon_small())
    np.testing.assert_array_equal(ion.kappa, g["kappa"])
    np.testing.assert_allclose(ion.P, g["P"], atol=1e-12)
    np.testing.assert_allclose(ion.Q, g["Q"], atol=1e-12)


def test_batch_ion_digests():
    from atomx_b200 import workloads as W
    g = np.load(os.path.join(GOLDEN, "batch_ions.npz"))
    specs = W.uneven_batch()
    for i in g["ions"]:
        assert W.build_ion(specs[int(i)]).coefficient_digest() == str(g[f"ion{int(i)}_digest"])


@pytest.mark.parametrize("name,pairs,rows,ordered", [
    ("neon_small", 10, 11, 45),
    ("ytterbium_scaleup", 20100, 56209, 318112753),
])
def test_plan_counts(name, pairs, rows, ordered):
    from atomx_b200 import plan as PL
    from atomx_b200 import workloads as W
    spec = getattr(W, name)()
    kap = np.concatenate([[k] * c for k, c in spec.shells])
    p = PL.make_plan(kap, spec.k_max)
    assert p.n_pairs == pairs and p.n_rows == rows
    assert p.ordered_entries == ordered


def test_allowed_k_rule():
    from atomx_b200.angular import exchange_k_range
    assert exchange_k_range(-1, -1) == [0]
    assert exchange_k_range(-1, 1) == [1]
    assert exchange_k_range(-1, -2) == [1]
    assert exchange_k_range(-2, -2) == [0, 2]
    assert exchange_k_range(2, -3) == [2, 4]  # d3/2 with d5/2: l=2,2 -> even k
    with pytest.raises(ValueError):
        exchange_k_range(0, 1)
