"""Host-side table plan: which pair densities and Y^k rows an ion needs.

A table entry R^k(ac;bd) = sum_i w_i rho_ac(r_i) Y^k[rho_bd](r_i) exists when
k is allowed for both unordered pairs (a, c) and (b, d)
(atomx angular/coefficients.py:186-210).  The plan

* enumerates unordered pairs (a <= c) grouped into kappa-pair blocks (all
  pairs whose spinors carry the same two kappas), blocks in shell order;
* lists, for every k, the pairs that allow it (``pairs_of_k[k]``, sorted by
  block so that each (k, block_ac, block_bd) tile is a contiguous rectangle
  of the k-th table);
* flattens (pair, k) into the Y^k / transform rows the device computes.

The k-th table is the symmetric n_k x n_k matrix over ``pairs_of_k[k]``;
ordered entries = sum_k n_k^2, unique entries = sum_k n_k (n_k + 1) / 2.
"""
from __future__ import annotations

from dataclasses import dataclass

import threading

import numpy as np

from .angular import exchange_k_range

__all__ = ["TablePlan", "make_plan"]


@dataclass
class TablePlan:
    kappa: np.ndarray          # (n_orb,) kappa of each spinor
    pairs: np.ndarray          # (n_pairs, 2) int64, a <= c, grouped by block
    pair_block: np.ndarray     # (n_pairs,) block id
    blocks: list               # [(kappa_a, kappa_c, start, stop)] ranges into ``pairs``
    ks: list                   # multipoles present
    pairs_of_k: dict           # k -> (n_k,) int64 pair indices, ascending
    row_pair: np.ndarray       # (n_rows,) pair index of each (pair, k) row
    row_k: np.ndarray          # (n_rows,) k of each row
    k_row_offset: dict         # k -> first row of that k (rows grouped by k)

    @property
    def n_pairs(self) -> int:
        return int(self.pairs.shape[0])

    @property
    def n_rows(self) -> int:
        return int(self.row_pair.shape[0])

    def n_of_k(self, k: int) -> int:
        return int(self.pairs_of_k[k].shape[0])

    @property
    def ordered_entries(self) -> int:
        return int(sum(self.n_of_k(k) ** 2 for k in self.ks))

    @property
    def unique_entries(self) -> int:
        return int(sum(self.n_of_k(k) * (self.n_of_k(k) + 1) // 2 for k in self.ks))

    def block_ranges_of_k(self, k: int):
        """[(block_id, start, stop)] row ranges of the k-th table."""
        bid = self.pair_block[self.pairs_of_k[k]]
        if bid.shape[0] == 0:
            return []
        starts = np.concatenate([[0], np.flatnonzero(bid[1:] != bid[:-1]) + 1])
        stops = np.concatenate([starts[1:], [bid.shape[0]]])
        return [(int(bid[a]), int(a), int(b)) for a, b in zip(starts, stops)]


_plan_cache: dict = {}
_plan_lock = threading.Lock()


def make_plan(kappa, k_max: int) -> TablePlan:
    """The table plan of an orbital set (see TablePlan); cached by the kappa
    sequence and k_max, since it depends on nothing else.  Plans are shared:
    treat their arrays as read-only."""
    kappa = np.asarray(kappa, dtype=np.int64)
    key = (kappa.tobytes(), int(k_max)) if kappa.ndim == 1 else None
    if key is not None:
        with _plan_lock:
            hit = _plan_cache.get(key)
        if hit is not None:
            return hit
    plan = _make_plan(kappa, k_max)
    if key is not None:
        for a in (plan.kappa, plan.pairs, plan.pair_block, plan.row_pair, plan.row_k, *plan.pairs_of_k.values()):
            a.setflags(write=False)
        with _plan_lock:
            if len(_plan_cache) > 1024:
                _plan_cache.clear()
            plan = _plan_cache.setdefault(key, plan)
    return plan


def _make_plan(kappa, k_max: int) -> TablePlan:
    n = kappa.shape[0]
    if n == 0:
        raise ValueError("an ion needs at least one spinor")
    if k_max < 0:
        raise ValueError("k_max must be a nonnegative integer")
    # Shells: maximal runs of equal kappa in orbital order.
    starts = [0] + [i for i in range(1, n) if kappa[i] != kappa[i - 1]]
    shells = [(int(kappa[s]), s, (starts[j + 1] if j + 1 < len(starts) else n)) for j, s in enumerate(starts)]
    pair_parts, block_parts, blocks, allowed_of_block = [], [], [], []
    count = 0
    for i, (ka, sa, ea) in enumerate(shells):
        for j in range(i, len(shells)):
            kc, sc, ec = shells[j]
            if i == j:  # a <= c within the shell, a-major order
                a, c = np.triu_indices(ea - sa)
                a, c = a + sa, c + sa
            else:
                a = np.repeat(np.arange(sa, ea), ec - sc)
                c = np.tile(np.arange(sc, ec), ea - sa)
            pair_parts.append(np.stack([a, c], axis=1))
            block_parts.append(np.full(a.shape[0], len(blocks), dtype=np.int64))
            blocks.append((ka, kc, count, count + a.shape[0]))
            count += a.shape[0]
            allowed_of_block.append([k for k in exchange_k_range(ka, kc) if k <= k_max])
    pairs = np.concatenate(pair_parts).astype(np.int64).reshape(-1, 2)
    pblock = np.concatenate(block_parts)
    ks = sorted({k for al in allowed_of_block for k in al})
    pairs_of_k = {}
    for k in ks:
        idx = [np.arange(b[2], b[3]) for bi, b in enumerate(blocks) if k in allowed_of_block[bi]]
        pairs_of_k[k] = np.concatenate(idx).astype(np.int64) if idx else np.zeros(0, np.int64)
    off, pos = {}, 0
    for k in ks:
        off[k] = pos
        pos += pairs_of_k[k].shape[0]
    row_pair = np.concatenate([pairs_of_k[k] for k in ks]) if ks else np.zeros(0, np.int64)
    row_k = np.concatenate([np.full(pairs_of_k[k].shape[0], k, dtype=np.int64) for k in ks]) if ks else \
        np.zeros(0, np.int64)
    return TablePlan(kappa=kappa, pairs=pairs, pair_block=pblock, blocks=blocks, ks=ks,
                     pairs_of_k=pairs_of_k, row_pair=row_pair.astype(np.int64), row_k=row_k, k_row_offset=off)
