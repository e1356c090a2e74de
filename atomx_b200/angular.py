"""Integer selection rules that decide which R^k table tiles exist.

Only the triangle and parity rules of the multipole expansion are needed on
this path: R^k(ab;cd) couples the pair densities rho_ac and rho_bd, and k is
allowed for a pair (a, c) when

    |j_a - j_c| <= k <= j_a + j_c   and   l_a + l_c + k is even,

the rule of atomx ``exchange_k_range`` (angular/coefficients.py:186-210) with
``l_of_kappa`` / ``twoj_of_kappa`` (angular/recoupling.py:113-132).  A table
entry R^k(ac;bd) exists when k is allowed for both pairs.
"""
from __future__ import annotations

__all__ = ["l_of_kappa", "twoj_of_kappa", "exchange_k_range", "kappa_label"]


def l_of_kappa(kappa: int) -> int:
    """Large-component orbital angular momentum: kappa<0 -> -kappa-1, kappa>0 -> kappa."""
    kappa = int(kappa)
    if kappa == 0:
        raise ValueError("kappa = 0 is not a valid relativistic quantum number")
    return -kappa - 1 if kappa < 0 else kappa


def twoj_of_kappa(kappa: int) -> int:
    """Twice the total angular momentum, 2|kappa| - 1."""
    kappa = int(kappa)
    if kappa == 0:
        raise ValueError("kappa = 0 is not a valid relativistic quantum number")
    return 2 * abs(kappa) - 1


def exchange_k_range(kappa_a: int, kappa_b: int) -> list[int]:
    """Multipoles k allowed between two spinors (triangle + parity)."""
    la, lb = l_of_kappa(kappa_a), l_of_kappa(kappa_b)
    ta, tb = twoj_of_kappa(kappa_a), twoj_of_kappa(kappa_b)
    lo, hi = abs(ta - tb) // 2, (ta + tb) // 2
    return [k for k in range(lo, hi + 1) if (k + la + lb) % 2 == 0]


_L_LETTERS = "spdfghiklmnoqrtuv"


def kappa_label(kappa: int) -> str:
    """Spectroscopic label such as 's1/2', 'p3/2' for a kappa."""
    return f"{_L_LETTERS[l_of_kappa(kappa)]}{twoj_of_kappa(kappa)}/2"
