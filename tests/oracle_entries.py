"""Sampled R^k entries from the oracle (the reference algorithm restated in
C), for device tests on inputs generated on the test host."""
import numpy as np

from oracle import oracle


def sampled_oracle_entries(ion, Pg, Qg, plan, per_k=32, seed=0):
    """Yield (k, i, j, R_ref) with i, j index arrays into the k-th table."""
    bd = ion.bsp
    gr, grw = bd["gr"], bd["grw"]
    nv, ng = gr.shape
    rng = np.random.default_rng(seed)
    for k in plan.ks:
        pk = plan.pairs_of_k[k]
        nk = pk.shape[0]
        ii = rng.integers(0, nk, size=per_k)
        jj = rng.integers(0, nk, size=per_k)
        # include the diagonal of every sampled row (Schwarz scale) and a corner
        ii = np.concatenate([ii, [0, nk - 1, nk - 1]])
        jj = np.concatenate([jj, [nk - 1, 0, nk - 1]])
        need = np.unique(np.concatenate([ii, jj]))
        pos = {int(p): t for t, p in enumerate(need)}
        rho = np.array([Pg[a] * Pg[c] + Qg[a] * Qg[c] for a, c in plan.pairs[pk[need]]])
        y = oracle.yk_rows(rho, k, gr, grw, nv, ng)
        g = rho * grw.reshape(1, -1)
        ia = np.array([pos[int(i)] for i in ii])
        ib = np.array([pos[int(j)] for j in jj])
        yield k, ii, jj, oracle.dot_entries(g, y, ia, ib)
