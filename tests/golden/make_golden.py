"""Generate the golden vectors that pin the oracle and the engine.

Run once, in a container where the atomx reference source is available:

    PYTHONPATH=<atomx>/src NUMBA_CACHE_DIR=/tmp/numba_cache \
        python tests/golden/make_golden.py --atomx-src <atomx>/src

It imports atomx's own functions (read-only) and writes small .npz fixtures
next to this script.  The fixtures are committed; the tests never import
atomx.  What each file holds:

* partial_matrices.npz   mo/mi of atomx ``yk_partial_matrices`` for several ng.
* neon_small.npz         the whole 1s/2s/2p1/2/2p3/2 Z=10 table (config of 40
                         order-7 splines): knots, grid, B-spline values,
                         atomx Dirac eigenvector coefficients, orbital node
                         values, every Y^k row, every ordered R^k entry via
                         ``slater_rk_poisson``, a few ``compute_slater_rk``
                         and ``slater_rk_direct`` values.
* ytterbium_scaleup.npz  Z=70, 200 rotated spinors: coefficient digest,
                         sampled Y^k rows with their densities, sampled R^k
                         entries.  (Spinors from LAPACK eigensolvers differ in
                         the last bits between hosts, so device tests use the
                         stored densities, not regenerated ones.)
* xenon_ci_table.npz     Z=54, 300 spinors, N=2112: digest, sampled entries.
* batch_ions.npz         three ions of the uneven batch: digests, samples.
* hydrogenic.npz         atomx physics grid (ks=9, Z=1, r_max=50): nodes and
                         weights, atomx R^k for rho = 4 r^2 e^{-2r} (k=0..2)
                         and rho = e^{-r} (k=0..3) with 40-digit mpmath values.
* direct_potential.npz   atomx DFSolver._build_direct_potential_yk
                         (methods/dirac_fock.py:931-967) run unmodified on a
                         stand-in ``self`` that carries only the attributes it
                         reads (bsp_data, ns, ks and the two grid evaluators):
                         the Z=10 ion with neon occupations and a 91-orbital
                         batch ion with seeded fractional occupations, each
                         with and without a target orbital.
                         (``--only direct`` writes just this file.)
* exchange_matrix.npz    atomx compute_exchange_matrix (numerics/bspline/
                         slater_yk.py:125, the rectangle-rule kernel :34-122)
                         for orbitals of the Z=10 ion and of a batch ion at
                         several k.  (``--only exchange`` writes just this file.)
* grid_quadrature.npz    atomx arbitrary-grid trapezoid Y^k (quadrature.py):
                         yk_on_grid / grid_slater_rk on a 1e-9..100 grid for
                         ranks up to 256, yk_pair_dot_batch_on_grid on the
                         reference's batch geometry and on a make_fine_grid
                         grid with seeded waves, and the endpoint cases.
                         (``--only grid`` writes just this file.)
* convol.npz             atomx's cell (bank) engine, numerics/bspline/convol.py:
                         whole banks on a tiny basis, cell Slater integrals
                         (scalar and batched), bilinear tables, direct and
                         exchange matrices and DBSR Fock blocks (see
                         ``convol_fixtures``).  (``--only convol``.)
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def grid_quadrature():
    """Golden vectors of atomx's arbitrary-grid trapezoid Y^k
    (numerics/quadrature.py): yk_on_grid, grid_slater_rk and
    yk_pair_dot_batch_on_grid on the reference's own test geometries plus a
    composite fine grid (make_fine_grid) with seeded random waves."""
    from atomx.numerics.quadrature import (grid_slater_rk, make_fine_grid, yk_on_grid,
                                           yk_pair_dot_batch_on_grid)
    out = {}
    # A: wide dynamic range, ranks up to 256
    r = np.geomspace(1e-9, 100.0, 193)
    rho = np.sin(3 * np.log(r)) * np.exp(-r / 12)
    other = np.cos(np.log(r)) * np.exp(-r / 9)
    ones, zeros = np.ones_like(r), np.zeros_like(r)
    ranks = np.array([0, 1, 12, 32, 64, 128, 256])
    out["a_r"], out["a_rho"], out["a_other"], out["a_ranks"] = r, rho, other, ranks
    out["a_yk"] = np.array([yk_on_grid(rho, r, int(k)) for k in ranks])
    out["a_yk_cut"] = np.array([yk_on_grid(rho, r, int(k), i_cut=97) for k in ranks])
    out["a_slater"] = np.array([grid_slater_rk(other, zeros, rho, zeros, ones, zeros, ones, zeros, r, int(k))
                                for k in ranks])
    # B: the batch geometry with invalid rows, empty and repeated consumers
    rng = np.random.default_rng(8217)
    rb = np.geomspace(.013, 9., 81)
    pa, qa, pb, qb = [rng.normal(size=(4, len(rb))) * np.exp(-rb / 4) for _ in range(4)]
    a, b = np.array([0, 2, 1, 3]), np.array([1, 0, 2, 0])
    rks, valid = np.array([0, 1, 3, 2]), np.array([True, True, False, True])
    ptr, cons = np.array([0, 2, 2, 5, 6]), np.array([0, 2, 1, 0, 3, 1])
    for cut in (0, 41, 80):
        outer = rng.normal(size=(4, cut + 1))
        out[f"b_outer{cut}"] = outer
        out[f"b_val{cut}"] = yk_pair_dot_batch_on_grid(pa, qa, pb, qb, a, b, rks, valid, outer, ptr, cons, rb,
                                                       i_cut=cut)
    out.update(b_r=rb, b_pa=pa, b_qa=qa, b_pb=pb, b_qb=qb, b_a=a, b_b=b, b_k=rks, b_ok=valid, b_ptr=ptr,
               b_cons=cons)
    # C: composite fine grid, seeded waves, many rows and consumers
    rf = np.asarray(make_fine_grid(30.0, 2.0, z_inner=20.0), dtype=float)
    rng = np.random.default_rng(4411)
    nw = 6
    env = np.exp(-rf / 6.0)
    P = rng.normal(size=(nw, rf.shape[0])) * env
    Q = 0.01 * rng.normal(size=(nw, rf.shape[0])) * env
    nrow = 24
    ra, rbb = rng.integers(0, nw, nrow), rng.integers(0, nw, nrow)
    rk_ = rng.integers(0, 9, nrow)
    ok = rng.random(nrow) > 0.1
    counts = rng.integers(0, 4, nrow)
    cptr = np.concatenate([[0], np.cumsum(counts)])
    ccons = rng.integers(0, 5, cptr[-1])
    cut = int(rf.shape[0] * 0.8)
    weights = rng.normal(size=(5, cut + 1)) * np.exp(-rf[:cut + 1] / 5.0)
    out.update(c_r=rf, c_P=P, c_Q=Q, c_a=ra, c_b=rbb, c_k=rk_, c_ok=ok, c_ptr=cptr, c_cons=ccons, c_w=weights,
               c_cut=np.array(cut))
    out["c_val"] = yk_pair_dot_batch_on_grid(P, Q, P, Q, ra, rbb, rk_, ok, weights, cptr, ccons, rf, i_cut=cut)
    out["c_slater"] = np.array([grid_slater_rk(P[0], Q[0], P[1], Q[1], P[2], Q[2], P[3], Q[3], rf, k)
                                for k in (0, 1, 4)])
    # D: endpoint rules (support cut with a half interval; a tiny far tail)
    r4 = np.array([0.1, 0.4, 1.0, 2.0])
    a4, b4, z4 = np.array([1.0, 2.0, 0.0, 0.0]), np.ones(4), np.zeros(4)
    r3 = np.array([1e-7, 1.0, 1e20])
    a3, b3, z3 = np.array([1.0, 1e-20, 1e-20]), np.ones(3), np.zeros(3)
    out["d_cut"] = np.array(grid_slater_rk(a4, z4, b4, z4, b4, z4, b4, z4, r4, 0))
    out["d_tail"] = np.array(grid_slater_rk(a3, z3, b3, z3, b3, z3, b3, z3, r3, 0))
    np.savez_compressed(os.path.join(HERE, "grid_quadrature.npz"), **out)


def direct_potential():
    """Inputs and outputs of atomx's direct-potential builder (see module doc)."""
    from types import MethodType, SimpleNamespace

    from atomx.methods.dirac_fock import DFSolver

    from atomx_b200 import workloads as W

    def run(ion, occ, target):
        bd = ion.bsp
        me = SimpleNamespace(bsp_data=bd, ns=int(bd["ns"]), ks=int(bd["ks"]))
        me._eval_P_on_grid = MethodType(DFSolver._eval_P_on_grid, me)
        me._eval_Q_on_grid = MethodType(DFSolver._eval_Q_on_grid, me)
        orbitals = {}
        for i, kappa in enumerate(ion.kappa):
            orbitals.setdefault(int(kappa), []).append((ion.P[i], ion.Q[i], float(occ[i])))
        plain = DFSolver._build_direct_potential_yk(me, orbitals)
        tk, ti = target
        minus = DFSolver._build_direct_potential_yk(me, orbitals, tk, ti)
        return plain, minus

    out = {}
    cases = {"neon": (W.build_ion(W.neon_small()), None, (-1, 1)),
             "batch5": (W.build_ion(W.uneven_batch()[5]), 7, (2, 3))}
    for name, (ion, seed, target) in cases.items():
        if seed is None:
            occ = np.array([2.0, 2.0, 2.0, 4.0])  # 1s2 2s2 2p1/2^2 2p3/2^4
        else:
            occ = np.random.default_rng(seed).uniform(0.0, 2.0, size=ion.kappa.shape[0])
        (vpp, vqq), (vpp_t, vqq_t) = run(ion, occ, target)
        bd = ion.bsp
        out.update({f"{name}_{k}": np.asarray(bd[k]) for k in ("gr", "grw", "bsp_p", "bsp_q")})
        out.update({f"{name}_{k}": int(bd[k]) for k in ("nv", "ks", "ksp", "ksq", "nsp", "nsq", "ns")})
        out.update({f"{name}_P": ion.P, f"{name}_Q": ion.Q, f"{name}_kappa": ion.kappa, f"{name}_occ": occ,
                    f"{name}_target": np.array(target), f"{name}_VPP": vpp, f"{name}_VQQ": vqq,
                    f"{name}_VPP_t": vpp_t, f"{name}_VQQ_t": vqq_t})
    np.savez_compressed(os.path.join(HERE, "direct_potential.npz"), **out)


def exchange_matrix():
    """Inputs and outputs of atomx compute_exchange_matrix (see module doc)."""
    from atomx.numerics.bspline.slater_yk import compute_exchange_matrix

    from atomx_b200 import workloads as W
    out = {}
    cases = {"neon": (W.build_ion(W.neon_small()), [(0, 0), (1, 1), (3, 2)]),
             "batch5": (W.build_ion(W.uneven_batch()[5]), [(0, 0), (17, 3), (60, 6)])}
    for name, (ion, picks) in cases.items():
        bd = ion.bsp
        out.update({f"{name}_{k}": np.asarray(bd[k]) for k in ("gr", "grw", "bsp_p", "bsp_q")})
        out.update({f"{name}_{k}": int(bd[k]) for k in ("nv", "ks", "ksp", "ksq", "nsp", "nsq", "ns")})
        out[f"{name}_picks"] = np.array(picks)
        for orb, k in picks:
            out[f"{name}_P{orb}"], out[f"{name}_Q{orb}"] = ion.P[orb], ion.Q[orb]
            kpp, kqq = compute_exchange_matrix(ion.P[orb], ion.Q[orb], bd, k)
            out[f"{name}_KPP_{orb}_{k}"], out[f"{name}_KQQ_{orb}_{k}"] = kpp, kqq
    np.savez_compressed(os.path.join(HERE, "exchange_matrix.npz"), **out)


def convol_fixtures():
    """Golden vectors of atomx's cell (bank) R^k engine, numerics/bspline/convol.py.

    Every input is stored with the outputs (basis arrays, coefficients), so
    the device tests run on exactly these numbers.

    * tiny: a 14-spline order-5 kinetically balanced basis on which whole
      banks fit a fixture: ConvolCache.get_rkb for all four component types at
      k = 0, 1, 3, and the local moments and diagonal-cell integrals behind
      them (_compute_moments_sym, _triang_sym / _triang_pqpq).
    * neon (the Z=10 ion, ns = 40 < SEMISEPARABLE_DIRECT_NS): 4-orbital keys
      through compute_slater_rk_cell (full-bank path) and
      compute_slater_rk_cell_batch; build_slater_rk_bilinear for one pair and
      compute_slater_rk_table over the four spinors; compute_direct_potential_cell
      and compute_exchange_matrix_cell at k = 0..2 (whole matrices at k = 1,
      seeded bra/ket projections at every k); the DBSR Fock blocks of
      DFSolver._build_hf_matrix_dbsr (methods/dirac_fock.py:1128) run
      unmodified on a stand-in ``self`` with seeded angular coefficients.
    * ytterbium (the Z=70 ion, ns = 120 >= SEMISEPARABLE_DIRECT_NS, whose scalar
      path is the factored one): seeded keys through compute_slater_rk_cell
      and compute_slater_rk_cell_batch, a bilinear table over 24 spinors, and
      projections of the direct and exchange matrices.
    """
    from types import MethodType, SimpleNamespace

    from atomx.methods.dirac_fock import DFSolver
    from atomx.numerics.bspline import convol as C

    from atomx_b200 import basis, workloads as W
    from atomx_b200.angular import exchange_k_range

    out = {}

    def keep_basis(name, bd):
        """The basis arrays themselves: a GPU host rebuilds nothing (its
        LAPACK and vector math may round differently in the last bit)."""
        out.update({f"{name}_{k}": np.asarray(bd[k]) for k in ("gr", "grw", "bsp_p", "bsp_q", "t", "tp")})
        out.update({f"{name}_{k}": int(bd[k]) for k in ("nv", "ks", "ksp", "ksq", "nsp", "nsq", "ns")})

    # --------------------------------------------------------------- tiny
    t = basis.make_exponential_knots(14, 5, 1e-4, 20.0)
    bd = basis.prepare_bspline_data(t, 14, 5, n_gauss=6, kinetic_balance=True)
    keep_basis("tiny", bd)
    cache = C.ConvolCache(bd)
    for k in (0, 1, 3):
        for itype in ("pppp", "qqqq", "pqpq", "qpqp"):
            rkb, ns, ks = cache.get_rkb(k, itype)
            out[f"tiny_rkb_{itype}_{k}"] = rkb
        for comp, ksx, b in (("p", bd["ksp"], bd["bsp_p"]), ("q", bd["ksq"], bd["bsp_q"])):
            out[f"tiny_rising_{comp}_{k}"] = C._compute_moments_sym(b, bd["gr"], bd["grw"], bd["nv"], ksx, k)
            out[f"tiny_falling_{comp}_{k}"] = C._compute_moments_sym(b, bd["gr"], bd["grw"], bd["nv"], ksx, -(k + 1))
        out[f"tiny_diag_pppp_{k}"] = C._triang_sym(bd["bsp_p"], bd["gr"], bd["grw"], bd["tp"], bd["nv"], bd["ksp"],
                                                   bd["ns"], k)
        out[f"tiny_diag_pqpq_{k}"] = C._triang_pqpq(bd["bsp_p"], bd["bsp_q"], bd["gr"], bd["grw"], bd["tp"], bd["t"],
                                                    bd["nv"], bd["ksp"], bd["ksq"], bd["ns"], k)
    cache.release_shared_banks()

    def keys_of(kappa, picks, rng, n_keys):
        keys = []
        while len(keys) < n_keys:
            a, b, c, d = (int(x) for x in rng.choice(picks, 4))
            ks = sorted(set(exchange_k_range(int(kappa[a]), int(kappa[b])))
                        & set(exchange_k_range(int(kappa[c]), int(kappa[d]))))
            if ks:
                keys.append((a, b, c, d, int(rng.choice(ks))))
        return np.array(keys, dtype=np.int64)

    def projections(ion, cache, name, ks_, rng, orbs):
        bd = ion.bsp
        ns = bd["ns"]
        vecs = rng.normal(size=(6, 2, ns))
        jp, kp = [], []
        for k in ks_:
            for slot, o in enumerate(orbs):
                J = C.compute_direct_potential_cell(ion.P[o], ion.Q[o], bd, k, cache=cache)
                K = C.compute_exchange_matrix_cell(ion.P[o], ion.Q[o], ion.P[o], ion.Q[o], bd, k, cache=cache)
                a, b = vecs[2 * slot], vecs[2 * slot + 1]
                jp.append((k, o, a[0] @ J[0] @ b[0], a[1] @ J[1] @ b[1]))
                kp.append((k, o, a[0] @ K[0] @ b[0], a[1] @ K[1] @ b[1], a[0] @ K[2] @ b[1], a[1] @ K[3] @ b[0]))
        out[f"{name}_proj_vecs"] = vecs
        out[f"{name}_direct_proj"] = np.array(jp)
        out[f"{name}_exchange_proj"] = np.array(kp)

    # --------------------------------------------------------------- neon
    ion = W.build_ion(W.neon_small())
    bd = ion.bsp
    keep_basis("neon", bd)
    out["neon_P"], out["neon_Q"], out["neon_kappa"] = ion.P, ion.Q, ion.kappa
    cache = C.ConvolCache(bd)
    od = {i: (ion.P[i], ion.Q[i]) for i in range(ion.P.shape[0])}
    rng = np.random.default_rng(2024)
    keys = []
    for a in range(4):
        for b in range(4):
            for c in range(4):
                for d in range(4):
                    ks = sorted(set(exchange_k_range(int(ion.kappa[a]), int(ion.kappa[b])))
                                & set(exchange_k_range(int(ion.kappa[c]), int(ion.kappa[d]))))
                    keys += [(a, b, c, d, k) for k in ks if k <= 2]
    keys = np.array(keys, dtype=np.int64)
    out["neon_keys"] = keys
    out["neon_cell"] = np.array([C.compute_slater_rk_cell(*od[a], *od[b], *od[c], *od[d], bd, int(k), cache=cache)
                                 for a, b, c, d, k in keys])
    out["neon_batch"] = np.array(C.compute_slater_rk_cell_batch(od, [tuple(int(x) for x in kk) for kk in keys], bd,
                                                                cache=cache))
    M = C.build_slater_rk_bilinear(ion.P[0], ion.Q[0], ion.P[1], ion.Q[1], bd, 1, cache=cache)
    for name, m in zip(("PP", "QQ", "PQ", "QP"), M):
        out[f"neon_bilinear_{name}"] = m
    out["neon_bilinear_table"] = C.compute_slater_rk_table(M, ion.P.T, ion.Q.T, ion.P.T, ion.Q.T)
    J = C.compute_direct_potential_cell(ion.P[1], ion.Q[1], bd, 1, cache=cache)
    K = C.compute_exchange_matrix_cell(ion.P[1], ion.Q[1], ion.P[2], ion.Q[2], bd, 1, cache=cache)
    out["neon_direct_PP"], out["neon_direct_QQ"] = J
    for name, m in zip(("PP", "QQ", "PQ", "QP"), K):
        out[f"neon_exchange_{name}"] = m
    projections(ion, cache, "neon", (0, 1, 2), rng, (0, 1, 2))
    # DBSR Fock blocks on a stand-in solver: only the attributes the method reads
    n = ion.P.shape[0]
    kmax = 2
    ad = rng.uniform(-1.0, 1.0, size=(n, n, kmax + 1)) * (rng.random((n, n, kmax + 1)) < 0.7)
    ax = rng.uniform(-1.0, 1.0, size=(n, n, kmax + 1)) * (rng.random((n, n, kmax + 1)) < 0.7)
    norms = rng.uniform(0.5, 2.0, size=n)
    shells = [SimpleNamespace(kappa=int(x)) for x in ion.kappa]
    me = SimpleNamespace(bsp_data=bd, subshells=shells, _angular_direct=ad, _angular_exchange=ax,
                         _angular_k_for_target=[tuple(range(kmax + 1))] * n)
    me._mean_field_divisor = lambda i: float(norms[i])
    orbitals = {}
    for i, kappa in enumerate(ion.kappa):
        orbitals.setdefault(int(kappa), []).append((ion.P[i], ion.Q[i], 1.0))
    hf = []
    for target in range(n):
        for skip in (False, True):
            hf.append(np.stack(DFSolver._build_hf_matrix_dbsr(me, target, orbitals, skip_pq_exchange=skip)))
    out["neon_hf_angular_direct"], out["neon_hf_angular_exchange"], out["neon_hf_norms"] = ad, ax, norms
    out["neon_hf"] = np.array(hf)  # (target, skip) -> PP, QQ, PQ, QP
    cache.release_shared_banks()

    # ---------------------------------------------------------- ytterbium
    ion = W.build_ion(W.ytterbium_scaleup())
    bd = ion.bsp
    keep_basis("yb", bd)
    cache = C.ConvolCache(bd)
    od = {i: (ion.P[i], ion.Q[i]) for i in range(ion.P.shape[0])}
    rng = np.random.default_rng(70)
    picks = np.arange(0, 200, 9)[:24]
    out["yb_orbitals"], out["yb_P"], out["yb_Q"] = picks, ion.P[picks], ion.Q[picks]
    keys = keys_of(ion.kappa, picks, rng, 160)
    keys = keys[np.isin(keys[:, 4], [0, 1, 2, 5, 12])][:96]
    out["yb_keys"] = keys
    out["yb_cell"] = np.array([C.compute_slater_rk_cell(*od[a], *od[b], *od[c], *od[d], bd, int(k), cache=cache)
                               for a, b, c, d, k in keys])
    out["yb_batch"] = np.array(C.compute_slater_rk_cell_batch(od, [tuple(int(x) for x in kk) for kk in keys], bd,
                                                              cache=cache))
    M = C.build_slater_rk_bilinear(ion.P[0], ion.Q[0], ion.P[9], ion.Q[9], bd, 2, cache=cache)
    cols = picks
    out["yb_table_cols"] = cols
    out["yb_bilinear_table"] = C.compute_slater_rk_table(M, ion.P[cols].T, ion.Q[cols].T, ion.P[cols].T,
                                                         ion.Q[cols].T)
    projections(ion, cache, "yb", (0, 2), rng, (0, 9, 18))
    cache.release_shared_banks()
    np.savez_compressed(os.path.join(HERE, "convol.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--atomx-src", required=True)
    ap.add_argument("--only", choices=["grid", "direct", "exchange", "convol"], default=None,
                    help="write only one fixture family (the others are left as they are)")
    args = ap.parse_args()
    sys.path.insert(0, args.atomx_src)
    sys.path.insert(0, REPO)
    if args.only == "grid":
        grid_quadrature()
        print("golden grid fixtures written to", HERE)
        return
    if args.only == "direct":
        direct_potential()
        print("golden direct-potential fixtures written to", HERE)
        return
    if args.only == "convol":
        convol_fixtures()
        print("golden cell-engine fixtures written to", HERE)
        return
    if args.only == "exchange":
        exchange_matrix()
        print("golden exchange-matrix fixtures written to", HERE)
        return

    from atomx.numerics.bspline.basis import prepare_bspline_data as ref_prepare
    from atomx.numerics.bspline.dirac_assembly import build_dirac_matrices, solve_dirac
    from atomx.numerics.bspline.evaluate import eval_P, eval_Q
    from atomx.numerics.bspline.knots import make_exponential_knots, make_physics_knots
    from atomx.numerics.bspline.slater import slater_rk_direct, slater_rk_poisson
    from atomx.numerics.bspline.slater_yk import compute_slater_rk
    from atomx.numerics.yk import compute_yk, yk_partial_matrices

    from atomx_b200 import plan as PL
    from atomx_b200 import workloads as W

    # ------------------------------------------------------------------ mo/mi
    pm = {}
    for ng in (2, 5, 7, 8, 9, 11, 17):
        mo, mi = yk_partial_matrices(ng)
        pm[f"mo{ng}"], pm[f"mi{ng}"] = mo, mi
    np.savez_compressed(os.path.join(HERE, "partial_matrices.npz"), **pm)

    # ------------------------------------------------------------ neon_small
    spec = W.neon_small()
    t = make_exponential_knots(spec.ns, spec.ks, spec.r_min, spec.r_max)
    bd = ref_prepare(t, spec.ns, spec.ks, n_gauss=spec.n_gauss, kinetic_balance=True)
    Ps, Qs, kap = [], [], []
    for kappa, count in spec.shells:
        H, S = build_dirac_matrices(bd["ns"], kappa, spec.Z, bd)
        res = solve_dirac(H, S, bd["ns"], kappa, nsp=bd["nsp"], nsq=bd["nsq"])
        for i in range(count):
            P, Q, _ = res.get_orbital(i)
            Ps.append(P), Qs.append(Q), kap.append(kappa)
    P, Q, kap = np.array(Ps), np.array(Qs), np.array(kap)
    Pg = np.array([eval_P(c, bd).ravel() for c in P])
    Qg = np.array([eval_Q(c, bd).ravel() for c in Q])
    plan = PL.make_plan(kap, spec.k_max)
    gr, grw, nv, ng = bd["gr"], bd["grw"], bd["nv"], spec.n_gauss
    rho = np.array([Pg[a] * Pg[c] + Qg[a] * Qg[c] for a, c in plan.pairs])
    rows = np.array([compute_yk(rho[p].reshape(nv, ng), gr, grw, nv, ng, int(k)).ravel()
                     for p, k in zip(plan.row_pair, plan.row_k)])
    ent = []  # (k, i_ac, i_bd, value) indices into pairs_of_k[k]
    for k in plan.ks:
        pk = plan.pairs_of_k[k]
        for i, pa in enumerate(pk):
            for j, pb in enumerate(pk):
                ent.append((k, i, j, slater_rk_poisson(rho[pa], rho[pb], gr, grw, nv, ng, k)))
    ent = np.array(ent)
    # compute_slater_rk(a,b,c,d): pairs (1,2) and (3,4)
    quads = np.array([(0, 0, 0, 0, 0), (0, 1, 0, 1, 0), (0, 2, 1, 3, 1), (2, 3, 2, 3, 2), (1, 1, 3, 3, 2), (0, 3, 1, 2, 1)])
    csr = np.array([compute_slater_rk(P[a], Q[a], P[b], Q[b], P[c], Q[c], P[d], Q[d], bd, int(k))
                    for a, b, c, d, k in quads])
    direct = np.array([(pa, pb, k, slater_rk_direct(rho[pa], rho[pb], gr, grw, k))
                       for pa, pb, k in [(0, 0, 0), (1, 4, 0), (2, 7, 1), (3, 9, 2), (9, 9, 2), (5, 6, 0)]])
    np.savez_compressed(os.path.join(HERE, "neon_small.npz"), t=t, gr=gr, grw=grw, bsp_p=bd["bsp_p"],
                        bsp_q=bd["bsp_q"], P=P, Q=Q, kappa=kap, Pg=Pg, Qg=Qg, pairs=plan.pairs,
                        row_pair=plan.row_pair, row_k=plan.row_k, yk_rows=rows, entries=ent,
                        quads=quads, compute_slater_rk=csr, direct=direct)

    # ------------------------------------------------ large ions: sampled
    def sampled(spec, fname, n_rows=12, n_ent=300, seed=7):
        ion = W.build_ion(spec)
        bd = ion.bsp
        gr, grw, nv, ng = bd["gr"], bd["grw"], bd["nv"], spec.n_gauss
        plan = PL.make_plan(ion.kappa, spec.k_max)
        Pg = np.array([eval_P(c, bd).ravel() for c in ion.P])
        Qg = np.array([eval_Q(c, bd).ravel() for c in ion.Q])
        rng = np.random.default_rng(seed)
        rsel = np.sort(rng.choice(plan.n_rows, size=min(n_rows, plan.n_rows), replace=False))
        yrows, rrho = [], []
        for q in rsel:
            a, c = plan.pairs[plan.row_pair[q]]
            rrho.append(Pg[a] * Pg[c] + Qg[a] * Qg[c])
            yrows.append(compute_yk(rrho[-1].reshape(nv, ng), gr, grw, nv, ng, int(plan.row_k[q])).ravel())
        ents = []
        for _ in range(n_ent):
            k = int(rng.choice(plan.ks))
            pk = plan.pairs_of_k[k]
            i, j = int(rng.integers(pk.shape[0])), int(rng.integers(pk.shape[0]))
            a, c = plan.pairs[pk[i]]
            b, d = plan.pairs[pk[j]]
            r13 = Pg[a] * Pg[c] + Qg[a] * Qg[c]
            r24 = Pg[b] * Pg[d] + Qg[b] * Qg[d]
            ents.append((k, i, j, slater_rk_poisson(r13, r24, gr, grw, nv, ng, k)))
        return dict(digest=np.array(ion.coefficient_digest()), row_index=rsel, yk_rows=np.array(yrows),
                    row_rho=np.array(rrho), row_k=plan.row_k[rsel], entries=np.array(ents))

    c2 = sampled(W.ytterbium_scaleup(), "ytterbium_scaleup.npz")
    np.savez_compressed(os.path.join(HERE, "ytterbium_scaleup.npz"), **c2)
    c5 = sampled(W.xenon_ci_table(), "xenon_ci_table.npz", n_rows=6, n_ent=200)
    np.savez_compressed(os.path.join(HERE, "xenon_ci_table.npz"), **c5)
    batch = W.uneven_batch()
    pick = [0, 1, 2]
    bdict = {}
    for i in pick:
        s = sampled(batch[i], "", n_rows=4, n_ent=80, seed=11 + i)
        for key, v in s.items():
            bdict[f"ion{i}_{key}"] = v
    bdict["ions"] = np.array(pick)
    np.savez_compressed(os.path.join(HERE, "batch_ions.npz"), **bdict)

    # ------------------------------------------------------------ hydrogenic
    import mpmath as mp
    th, nsh = make_physics_knots(ks=9, Z=1, r_max=50.0)
    bdh = ref_prepare(th, nsh, 9)
    grh, grwh, nvh = bdh["gr"], bdh["grw"], bdh["nv"]
    rho1s = 4.0 * grh ** 2 * np.exp(-2.0 * grh)
    h1s = np.array([float(np.sum(grwh * rho1s * compute_yk(rho1s, grh, grwh, nvh, 9, k))) for k in (0, 1, 2)])
    # e^{-r} density on the same grid, with 40-digit references
    mp.mp.dps = 40
    expo, expo_ref = [], []
    rexp = np.exp(-grh)
    for k in (0, 1, 2, 3):
        expo.append(float(np.sum(grwh * rexp * compute_yk(rexp, grh, grwh, nvh, 9, k))))

        def yk_ref(rv, k=k):
            r = mp.mpf(rv)
            return (mp.gammainc(k + 1, 0, r) + r ** (2 * k + 1) * mp.quad(lambda s: mp.exp(-s) / s ** (k + 1), [r, mp.inf])) / r ** (k + 1)

        expo_ref.append(float(mp.quad(lambda r: mp.exp(-r) * yk_ref(r), [0, 1, 3, 10, mp.inf])))
    np.savez_compressed(os.path.join(HERE, "hydrogenic.npz"), t=th, gr=grh, grw=grwh, h1s=h1s,
                        expo=np.array(expo), expo_ref=np.array(expo_ref))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
