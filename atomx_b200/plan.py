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


def _triu_rows(l: np.ndarray, n: np.ndarray):
    """(row, col) of position l in the a-major upper triangle (diagonal
    included) of an n x n block: row i starts at i n - i (i - 1) / 2."""
    b = 2 * n + 1
    i = np.floor((b - np.sqrt(b.astype(np.float64) ** 2 - 8.0 * l)) / 2.0).astype(np.int64)
    for _ in range(2):  # guard the square root's rounding
        start = i * n - i * (i - 1) // 2
        i = np.where(start > l, i - 1, i)
        nxt = (i + 1) * n - (i + 1) * i // 2
        i = np.where(nxt <= l, i + 1, i)
    start = i * n - i * (i - 1) // 2
    return i, i + (l - start)


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
    same = si == sj
    na, nc = sizes[si], sizes[sj]
    bsize = np.where(same, na * (na + 1) // 2, na * nc)
    boff = np.concatenate([[0], np.cumsum(bsize)]).astype(np.int64)
    total = int(boff[-1])
    bid = np.repeat(np.arange(si.shape[0]), bsize)
    loc = np.arange(total, dtype=np.int64) - boff[bid]
    ncb = nc[bid]
    a_loc, c_loc = loc // ncb, loc % ncb
    sm = same[bid]
    if sm.any():
        a_loc[sm], c_loc[sm] = _triu_rows(loc[sm], na[bid][sm])
    pairs = np.stack([starts[si][bid] + a_loc, starts[sj][bid] + c_loc], axis=1).astype(np.int64)
    pblock = bid.astype(np.int64)
    allowed = np.array([_allowed_mask(int(skap[a]), int(skap[b]), int(k_max)) for a, b in zip(si, sj)],
                       dtype=bool).reshape(si.shape[0], k_max + 1)
    blocks = [(int(skap[a]), int(skap[b]), int(boff[t]), int(boff[t + 1])) for t, (a, b) in enumerate(zip(si, sj))]
    ks = [int(k) for k in np.flatnonzero(allowed.any(axis=0))]
    pairs_of_k = {k: np.flatnonzero(allowed[pblock, k]).astype(np.int64) for k in ks}
    off, pos = {}, 0
    for k in ks:
        off[k] = pos
        pos += pairs_of_k[k].shape[0]
    row_pair = np.concatenate([pairs_of_k[k] for k in ks]) if ks else np.zeros(0, np.int64)
    row_k = np.concatenate([np.full(pairs_of_k[k].shape[0], k, dtype=np.int64) for k in ks]) if ks else \
        np.zeros(0, np.int64)
    return TablePlan(kappa=kappa, pairs=pairs, pair_block=pblock, blocks=blocks, ks=ks,
                     pairs_of_k=pairs_of_k, row_pair=row_pair.astype(np.int64), row_k=row_k, k_row_offset=off)
