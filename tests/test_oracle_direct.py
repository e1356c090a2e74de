"""The oracle's direct potential (DFSolver._build_direct_potential_yk,
methods/dirac_fock.py:931-967) against atomx's own outputs on stored inputs.

The oracle evaluates the orbitals, accumulates the density and sums the
B-spline matrix in atomx's order with separately rounded operations, and
equals atomx bit for bit.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle


def _case(g, name):
    keys = ("gr", "grw", "bsp_p", "bsp_q", "nv", "ks", "ksp", "ksq", "nsp", "nsq", "ns")
    bd = {k: (g[f"{name}_{k}"] if g[f"{name}_{k}"].ndim else int(g[f"{name}_{k}"])) for k in keys}
    orbitals = {}
    for P, Q, kappa, occ in zip(g[f"{name}_P"], g[f"{name}_Q"], g[f"{name}_kappa"], g[f"{name}_occ"]):
        orbitals.setdefault(int(kappa), []).append((P, Q, float(occ)))
    return bd, orbitals, tuple(int(x) for x in g[f"{name}_target"])


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(GOLDEN, "direct_potential.npz"))


def _close(got, ref):
    assert got.shape == ref.shape
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("name", ["neon", "batch5"])
def test_oracle_direct_potential_matches_atomx(g, name):
    bd, orbitals, (tk, ti) = _case(g, name)
    vpp, vqq = oracle.direct_potential_yk(bd, bd["ns"], orbitals)
    _close(vpp, g[f"{name}_VPP"])
    _close(vqq, g[f"{name}_VQQ"])
    vpp_t, vqq_t = oracle.direct_potential_yk(bd, bd["ns"], orbitals, tk, ti)
    _close(vpp_t, g[f"{name}_VPP_t"])
    _close(vqq_t, g[f"{name}_VQQ_t"])
    # the target's own density is really taken out
    assert np.abs(vpp_t - vpp).max() > 1e-3 * np.abs(vpp).max()
    # symmetric, banded
    assert np.array_equal(vpp, vpp.T)
    ks = bd["ksp"]
    i, j = np.indices(vpp.shape)
    assert np.all(vpp[np.abs(i - j) >= ks] == 0.0)
