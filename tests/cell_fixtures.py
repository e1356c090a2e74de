"""Inputs of the cell-engine golden fixtures (tests/golden/convol.npz): the
stored basis arrays and coefficients, so that every host runs on exactly the
numbers atomx saw."""
import os

import numpy as np

from conftest import GOLDEN

_ARRAYS = ("gr", "grw", "bsp_p", "bsp_q", "t", "tp")
_INTS = ("nv", "ks", "ksp", "ksq", "nsp", "nsq", "ns")


def load():
    return np.load(os.path.join(GOLDEN, "convol.npz"))


def basis(g, name: str) -> dict:
    bd = {k: np.asarray(g[f"{name}_{k}"]) for k in _ARRAYS}
    bd.update({k: int(g[f"{name}_{k}"]) for k in _INTS})
    return bd


def orbitals(g, name: str) -> dict:
    """{orbital index: (P, Q)} of the stored spinors."""
    if name == "neon":
        return {i: (g["neon_P"][i], g["neon_Q"][i]) for i in range(g["neon_P"].shape[0])}
    return {int(o): (g["yb_P"][r], g["yb_Q"][r]) for r, o in enumerate(g["yb_orbitals"])}
