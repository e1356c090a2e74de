"""The oracle's exchange matrices (compute_exchange_matrix, atomx
numerics/bspline/slater_yk.py:125 with the rectangle-rule kernel :34-122)
equal atomx's outputs bit for bit on stored inputs."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle


def exchange_case(g, name):
    keys = ("gr", "grw", "bsp_p", "bsp_q", "nv", "ks", "ksp", "ksq", "nsp", "nsq", "ns")
    bd = {k: (g[f"{name}_{k}"] if g[f"{name}_{k}"].ndim else int(g[f"{name}_{k}"])) for k in keys}
    return bd, [(int(o), int(k)) for o, k in g[f"{name}_picks"]]


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(GOLDEN, "exchange_matrix.npz"))


@pytest.mark.parametrize("name", ["neon", "batch5"])
def test_oracle_exchange_matrix_matches_atomx(g, name):
    bd, picks = exchange_case(g, name)
    for orb, k in picks:
        kpp, kqq = oracle.compute_exchange_matrix(g[f"{name}_P{orb}"], g[f"{name}_Q{orb}"], bd, k)
        np.testing.assert_array_equal(kpp, g[f"{name}_KPP_{orb}_{k}"])
        np.testing.assert_array_equal(kqq, g[f"{name}_KQQ_{orb}_{k}"])
        assert kpp.shape == (bd["nsp"], bd["nsp"]) and kqq.shape == (bd["nsq"], bd["nsq"])
