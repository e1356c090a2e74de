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
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--atomx-src", required=True)
    args = ap.parse_args()
    sys.path.insert(0, args.atomx_src)
    sys.path.insert(0, REPO)

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
