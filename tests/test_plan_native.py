"""The native table-plan builder (rkb_table_plan behind plan.make_plan)
against a whole-array numpy restatement of the same plan: identical pairs,
blocks, multipoles, per-k pair lists and rows, on the serving stream's
orbital sets and on random kappa sequences (repeated and interleaved
shells, one spinor, k_max 0)."""
import numpy as np
import pytest

from atomx_b200 import plan as PL


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


def _plan_reference(kappa, k_max: int):
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
    allowed = np.array([PL._allowed_mask(int(skap[a]), int(skap[b]), int(k_max)) for a, b in zip(si, sj)],
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
    return dict(pairs=pairs, pair_block=pblock, blocks=blocks, ks=ks, pairs_of_k=pairs_of_k,
                row_pair=row_pair.astype(np.int64), row_k=row_k, k_row_offset=off)


def _check(kappa, k_max):
    kappa = np.asarray(kappa, dtype=np.int64)
    got = PL._make_plan(kappa, k_max)
    want = _plan_reference(kappa, k_max)
    assert np.array_equal(got.pairs, want["pairs"]) and got.pairs.dtype == np.int64
    assert np.array_equal(got.pair_block, want["pair_block"])
    assert got.blocks == want["blocks"] and got.ks == want["ks"] and got.k_row_offset == want["k_row_offset"]
    assert np.array_equal(got.row_pair, want["row_pair"]) and np.array_equal(got.row_k, want["row_k"])
    assert sorted(got.pairs_of_k) == sorted(want["pairs_of_k"])
    for k, v in want["pairs_of_k"].items():
        assert np.array_equal(got.pairs_of_k[k], v)


def test_serving_orbital_sets():
    from atomx_b200 import workloads as W
    for _, spec in W.serving_requests(n_requests=24):
        _check(W.build_ion(spec).kappa, spec.k_max)


@pytest.mark.parametrize("seed", range(8))
def test_random_kappa_sequences(seed):
    rng = np.random.default_rng(seed)
    choices = np.array([-1, 1, -2, 2, -3, 3, -4, 4, -5, 5, -6, 6, -7, 7])
    for n in (1, 2, 5, 17, 60):
        kappa = rng.choice(choices[:int(rng.integers(1, 15))], n)
        if seed % 2:
            kappa = np.sort(kappa)  # long shells
        for k_max in (0, 3, 12):
            _check(kappa, k_max)
