"""Accuracy probes of whole R^k tables against the oracle — TEST INFRASTRUCTURE ONLY.

Used by the device tests and by the benchmark's CPU-baseline leg, as the
checker.  The engine never imports it.

Two error metrics of a table entry R(ac;bd) against the reference value:

* floored relative: |x - ref| / max(|ref|, 1e-6 max|ref|), the max taken over
  the multipole table;
* Schwarz relative: |x - ref| / sqrt(|ref(ac;ac)| |ref(bd;bd)|), the entry's
  Cauchy-Schwarz scale (R^k is an inner product in the positive Coulomb
  metric, so |R(ac;bd)| never exceeds it).

The floored metric is largest where an entry is much smaller than its
Schwarz scale (a cancelling entry), so a uniform random sample of a large
table rarely meets its worst case.  ``probe_entries`` therefore takes the
entries of largest sensitivity scale / max(|R|, floor) of a table computed on
the device, plus seeded random ones, and ``oracle_entries`` evaluates them by
the reference algorithm: Y^k of the bd density (atomx numerics/yk.py:88-154,
``oracle.yk_rows``) and one quadrature dot per entry (numerics/bspline/
slater.py:130, ``oracle.dot_entries``).  It also evaluates every entry the
other way round, R(bd;ac) as the reference would compute it with the pairs
exchanged, which measures how far the reference's own two evaluations of one
integral differ.
"""
from __future__ import annotations

import numpy as np

from . import oracle

FLOOR = 1e-6


def probe_entries(table, n_cand: int = 2048, n_rand: int = 2048, seed: int = 0):
    """(ii, jj) index arrays into an n x n device table (torch tensor): the
    n_cand entries of largest sensitivity sqrt|T_ii T_jj| / max(|T_ij|,
    1e-6 max|T|), then n_rand seeded random entries."""
    import torch
    n = table.shape[0]
    a = table.abs()
    d = torch.diagonal(table).abs().sqrt()
    floor = FLOOR * float(a.max())
    sens = torch.outer(d, d) / a.clamp_min(floor)
    c = min(n_cand, n * n)
    idx = torch.topk(sens.reshape(-1), c).indices.cpu().numpy()
    rng = np.random.default_rng(seed)
    rnd = rng.integers(0, n * n, size=n_rand)
    idx = np.concatenate([idx, rnd]).astype(np.int64)
    return idx // n, idx % n


def oracle_entries(plan, k, ii, jj, Pg, Qg, gr, grw, threads: int = 0):
    """Reference values at entries (ii, jj) of the k-th table: R(ii;jj), the
    same integral with the pairs exchanged R(jj;ii), and the diagonal
    R(p;p) of every row p of the table (for the Schwarz scale and the
    table's floor).  Pg, Qg: orbital values on the (nv, ng) grid."""
    nv, ng = gr.shape
    pk = plan.pairs[plan.pairs_of_k[k]]
    rho = Pg[pk[:, 0]] * Pg[pk[:, 1]] + Qg[pk[:, 0]] * Qg[pk[:, 1]]
    y = oracle.yk_rows(rho, k, gr, grw, nv, ng, threads=threads)
    g = rho * np.asarray(grw).reshape(1, -1)
    n = pk.shape[0]
    diag = oracle.dot_entries(g, y, np.arange(n), np.arange(n), threads=threads)
    fwd = oracle.dot_entries(g, y, ii, jj, threads=threads)
    rev = oracle.dot_entries(g, y, jj, ii, threads=threads)
    return fwd, rev, diag


def entry_errors(got, ref, ii, jj, diag, table_max):
    """Floored-relative, Schwarz-relative and absolute errors of ``got``
    against ``ref`` at entries (ii, jj); NaNs count as infinite."""
    got = np.asarray(got, dtype=np.float64)
    d = np.abs(got - ref)
    d = np.where(np.isnan(d), np.inf, d)
    scale = np.sqrt(np.abs(diag[ii]) * np.abs(diag[jj]))
    floored = d / np.maximum(np.abs(ref), FLOOR * table_max)
    schwarz = d / scale
    return {"rel_floored_1e-6": float(floored.max()) if d.size else 0.0,
            "schwarz_rel": float(schwarz.max()) if d.size else 0.0,
            "abs": float(d.max()) if d.size else 0.0}
