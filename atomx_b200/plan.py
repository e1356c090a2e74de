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

import threading
from dataclasses import dataclass
from functools import lru_cache

import numpy as np

from . import _native

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
        """[(block_id, start, stop)] row ranges of the k-th table (computed
        once per plan and k; a fresh list each call)."""
        cache = self.__dict__.setdefault("_block_ranges", {})
        hit = cache.get(k)
        if hit is None:
            bid = self.pair_block[self.pairs_of_k[k]]
            if bid.shape[0] == 0:
                hit = ()
            else:
                starts = np.concatenate([[0], np.flatnonzero(bid[1:] != bid[:-1]) + 1])
                stops = np.concatenate([starts[1:], [bid.shape[0]]])
                hit = tuple(zip(bid[starts].tolist(), starts.tolist(), stops.tolist()))
            cache[k] = hit
        return list(hit)


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


@lru_cache(maxsize=4096)
def _allowed_mask(kappa_a: int, kappa_c: int, k_max: int) -> tuple:
    """k <= k_max allowed for a pair of these kappas, as a tuple of bools."""
    al = set(exchange_k_range(kappa_a, kappa_c))
    return tuple(k in al for k in range(k_max + 1))


def _make_plan(kappa, k_max: int) -> TablePlan:
    n = kappa.shape[0]
    if n == 0:
        raise ValueError("an ion needs at least one spinor")
    if k_max < 0:
        raise ValueError("k_max must be a nonnegative integer")
    # Shells: maximal runs of equal kappa in orbital order.
    cut = np.flatnonzero(kappa[1:] != kappa[:-1]) + 1
    starts = np.concatenate([[0], cut]).astype(np.int64)
    sizes = np.diff(np.concatenate([starts, [n]])).astype(np.int64)
    skap = kappa[starts]
    # Blocks: shell pairs (i <= j) in i-major order; pairs a <= c within a shell, a-major.
    si, sj = np.triu_indices(starts.shape[0])
    na, nc = sizes[si], sizes[sj]
    bsize = np.where(si == sj, na * (na + 1) // 2, na * nc)
    boff = np.concatenate([[0], np.cumsum(bsize)]).astype(np.int64)
    allowed = np.array([_allowed_mask(a, c, int(k_max)) for a, c in zip(skap[si].tolist(), skap[sj].tolist())],
                       dtype=np.uint8).reshape(si.shape[0], k_max + 1)
    per_k = bsize @ allowed.astype(np.int64)             # rows of each k
    ks = np.flatnonzero(per_k).tolist()
    n_pairs, n_rows = int(boff[-1]), int(per_k.sum())
    pairs = np.empty((n_pairs, 2), dtype=np.int64)
    pblock = np.empty(n_pairs, dtype=np.int64)
    row_pair = np.empty(n_rows, dtype=np.int64)
    row_k = np.empty(n_rows, dtype=np.int64)
    allowed = np.ascontiguousarray(allowed)
    # the pair and row arrays, filled natively (no interpreter lock held)
    got = _native.load().rkb_table_plan(starts.ctypes.data, sizes.ctypes.data, int(starts.shape[0]),
                                        allowed.ctypes.data, int(k_max), n_pairs, n_rows, pairs.ctypes.data,
                                        pblock.ctypes.data, row_pair.ctypes.data, row_k.ctypes.data)
    if got < 0:
        _native.check(int(-got), "rkb_table_plan")
    blocks = list(zip(skap[si].tolist(), skap[sj].tolist(), boff[:-1].tolist(), boff[1:].tolist()))
    off, pairs_of_k, pos = {}, {}, 0
    for k in ks:
        off[k] = pos
        pairs_of_k[k] = row_pair[pos:pos + int(per_k[k])]
        pos += int(per_k[k])
    return TablePlan(kappa=kappa, pairs=pairs, pair_block=pblock, blocks=blocks, ks=ks,
                     pairs_of_k=pairs_of_k, row_pair=row_pair, row_k=row_k, k_row_offset=off)
