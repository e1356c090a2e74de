"""CPU oracle for the R^k / Y^k path — TEST INFRASTRUCTURE ONLY.

Only the test-suite, ``__graft_entry__.smoke()`` (as the checker) and the
benchmark's CPU-baseline leg import this module.  The engine never does.

Each function restates the reference algorithm (atomx; paths are relative to
its project root) in plain numpy or calls the C restatement in
``rk_oracle.c``:

* ``yk_partial_matrices``   <- src/atomx/numerics/yk.py:65-84
* ``yk_rows`` / ``yk_row``  <- src/atomx/numerics/yk.py:88-154 (C, bit-faithful)
* ``eval_orbital_on_grid``  <- src/atomx/numerics/bspline/evaluate.py:71-97
* ``pair_density``          <- src/atomx/numerics/bspline/slater_yk.py:193-194
* ``slater_rk_poisson``     <- src/atomx/numerics/bspline/slater.py:118-130
* ``slater_rk_direct``      <- src/atomx/numerics/bspline/slater.py:51-115
* ``dot_entries``           <- slater.py:130, one dot per ordered table entry
* ``coulomb_tables``        <- src/atomx/numerics/quadrature.py:190-231 (numpy)
* ``yk_on_grid`` / ``grid_slater_rk`` / ``yk_pair_dot_batch_on_grid``
                            <- quadrature.py:234-404 (C, bit-faithful)
* ``direct_potential_yk``   <- src/atomx/methods/dirac_fock.py:931-967 with
                               numerics/bspline/integrals.py:18-56 (C)
* ``compute_exchange_matrix`` <- src/atomx/numerics/bspline/slater_yk.py:34-155 (C)

Parity of the oracle itself is pinned against vectors generated by running
the reference (tests/golden/make_golden.py) and against closed forms.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from functools import lru_cache

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "librk_oracle.so")

_dptr = ctypes.POINTER(ctypes.c_double)
_iptr = ctypes.POINTER(ctypes.c_int)
_lptr = ctypes.POINTER(ctypes.c_long)


def build() -> str:
    """Compile the C oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


@lru_cache(maxsize=1)
def _lib():
    if not os.path.exists(_LIB_PATH) or any(
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, src))
            for src in ("rk_oracle.c", "cell_oracle.c")):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    lib.oracle_yk_rows.argtypes = [_dptr, _iptr, ctypes.c_long, _dptr, _dptr, ctypes.c_int,
                                   ctypes.c_int, _dptr, _dptr, _dptr, ctypes.c_int]
    lib.oracle_yk_rows.restype = None
    lib.oracle_dot_table.argtypes = [_dptr, _dptr, ctypes.c_long, _lptr, _lptr, ctypes.c_long,
                                     _dptr, ctypes.c_int]
    lib.oracle_dot_table.restype = None
    lib.oracle_dot_block.argtypes = [_dptr, ctypes.c_long, _dptr, ctypes.c_long, ctypes.c_long, _dptr,
                                     ctypes.c_int]
    lib.oracle_dot_block.restype = None
    lib.oracle_int_pow.argtypes = [ctypes.c_double, ctypes.c_long]
    lib.oracle_int_pow.restype = ctypes.c_double
    lib.oracle_max_threads.restype = ctypes.c_int
    return lib


def max_threads() -> int:
    return int(_lib().oracle_max_threads())


def _p(a, ptr=_dptr):
    return a.ctypes.data_as(ptr)


@lru_cache(maxsize=32)
def yk_partial_matrices(ng: int):
    """Interpolatory partial-cell matrices (mo, mi = 1 - mo) for ``ng`` nodes.

    mo[i, j] * w_j is the integral of the j-th Lagrange basis polynomial from
    the cell's left edge to node i, evaluated through the orthogonal Legendre
    expansion L_j(x)/w_j = sum_l (2l+1)/2 P_l(x_j) P_l(x) and the antiderivative
    identity int_{-1}^x P_l = (P_{l+1} - P_{l-1})/(2l+1) (int P_0 = x + 1).
    """
    xi, _ = np.polynomial.legendre.leggauss(ng)
    vand = np.polynomial.legendre.legvander(xi, ng)  # P_0..P_ng at the nodes
    anti = np.empty((ng, ng))
    anti[:, 0] = xi + 1.0
    for ell in range(1, ng):
        anti[:, ell] = (vand[:, ell + 1] - vand[:, ell - 1]) / (2 * ell + 1)
    mo = (anti * ((2 * np.arange(ng) + 1) / 2.0)) @ vand[:, :ng].T
    mo.setflags(write=False)
    mi = 1.0 - mo
    mi.setflags(write=False)
    return mo, mi


def yk_rows(rho: np.ndarray, ks, r: np.ndarray, w: np.ndarray, nv: int, ng: int,
            threads: int = 0) -> np.ndarray:
    """Y^k rows: ``rho`` is (nrows, nv*ng); ``ks`` a scalar or (nrows,) ints."""
    rho = np.ascontiguousarray(np.atleast_2d(rho), dtype=np.float64)
    nrows, n = rho.shape
    assert n == nv * ng
    ks = np.ascontiguousarray(np.broadcast_to(np.asarray(ks, dtype=np.int32), (nrows,)))
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1)
    w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
    mo, mi = yk_partial_matrices(ng)
    mo = np.ascontiguousarray(mo)
    mi = np.ascontiguousarray(mi)
    out = np.empty_like(rho)
    _lib().oracle_yk_rows(_p(rho), _p(ks, _iptr), nrows, _p(r), _p(w), nv, ng, _p(mo), _p(mi),
                          _p(out), int(threads))
    return out


def yk_row(rho, r, w, nv, ng, k):
    return yk_rows(np.asarray(rho).reshape(1, -1), k, r, w, nv, ng, threads=1)[0]


def dot_entries(g: np.ndarray, y: np.ndarray, ia, ib, threads: int = 0) -> np.ndarray:
    """out[e] = g[ia[e]] . y[ib[e]] with one plain dot per entry."""
    g = np.ascontiguousarray(g, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    ia = np.ascontiguousarray(ia, dtype=np.int64)
    ib = np.ascontiguousarray(ib, dtype=np.int64)
    out = np.empty(ia.shape[0])
    _lib().oracle_dot_table(_p(g), _p(y), g.shape[1], _p(ia, _lptr), _p(ib, _lptr), ia.shape[0],
                            _p(out), int(threads))
    return out


def dot_block(g: np.ndarray, y: np.ndarray, threads: int = 0, out: np.ndarray | None = None) -> np.ndarray:
    """out[j, i] = g[i] . y[j]: every row of g against every row of y, one
    plain dot per entry (the per-integral sum of slater_rk_poisson)."""
    g = np.ascontiguousarray(g, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    assert g.shape[1] == y.shape[1]
    if out is None:
        out = np.empty((y.shape[0], g.shape[0]))
    assert out.shape == (y.shape[0], g.shape[0]) and out.flags.c_contiguous and out.dtype == np.float64
    _lib().oracle_dot_block(_p(g), g.shape[0], _p(y), y.shape[0], g.shape[1], _p(out), int(threads))
    return out


def eval_orbital_on_grid(coeffs: np.ndarray, bsp: np.ndarray, nv: int, ks: int, ns: int) -> np.ndarray:
    """f(r_im) = sum_s c[i+s] B_s(r_im) with coefficients beyond ns taken as 0."""
    coeffs = np.asarray(coeffs, dtype=np.float64)
    idx = np.arange(nv)[:, None] + np.arange(ks)[None, :]
    c = np.where(idx < ns, coeffs[np.minimum(idx, ns - 1)], 0.0)
    return np.einsum("is,ims->im", c, bsp)


def eval_P(coeffs, bsp_data):
    return eval_orbital_on_grid(coeffs, bsp_data["bsp_p"], bsp_data["nv"], bsp_data["ksp"], bsp_data["nsp"])


def eval_Q(coeffs, bsp_data):
    return eval_orbital_on_grid(coeffs, bsp_data["bsp_q"], bsp_data["nv"], bsp_data["ksq"], bsp_data["nsq"])


def pair_density(Pa, Qa, Pc, Qc):
    """Dirac pair density rho_ac = P_a P_c + Q_a Q_c (node values)."""
    return Pa * Pc + Qa * Qc


def slater_rk_poisson(rho13, rho24, gr, grw, nv, ng, k):
    rho24 = np.asarray(rho24, dtype=np.float64).reshape(nv, ng)
    rho13 = np.asarray(rho13, dtype=np.float64).reshape(nv, ng)
    y = yk_row(rho24, gr, grw, nv, ng, k).reshape(nv, ng)
    return float(np.sum(grw * rho13 * y))


def _disjoint_cells(rho13, rho24, r, w, k, ng):
    """Product rule over cell pairs (m < m'), both orderings, vectorised."""
    n = r.shape[0]
    cell = np.arange(n) // ng
    later = cell[None, :] > cell[:, None]
    with np.errstate(over="ignore", under="ignore", invalid="ignore"):
        ker = np.where(later, (r[:, None] / r[None, :]) ** k / r[None, :], 0.0)
    prod = w[:, None] * w[None, :] * ker * (rho13[:, None] * rho24[None, :] + rho13[None, :] * rho24[:, None])
    return float(np.sum(prod))


@lru_cache(maxsize=16)
def _triangle_rule(ng, order):
    nodes, _ = np.polynomial.legendre.leggauss(ng)
    x, wt = np.polynomial.legendre.leggauss(order)
    x, wt = (x + 1.0) / 2.0, wt / 2.0
    inv = np.linalg.solve(np.polynomial.legendre.legvander(nodes, ng - 1), np.eye(ng))
    outer = np.polynomial.legendre.legvander(2 * x - 1, ng - 1) @ inv
    inner = np.polynomial.legendre.legvander(2 * x[:, None] * x[None, :] - 1, ng - 1) @ inv
    return nodes, x, wt, outer, inner


def slater_rk_direct(rho13, rho24, gr, grw, k):
    """O(N^2) double quadrature with each coincident cell split along r = s.

    Disjoint cell pairs use the tensor Gauss rule; a coincident cell uses the
    Duffy-type map r = a + h x, s = a + h x y on its lower triangle with a
    Gauss rule of order max(2 ng, (k + ng + 1)//2) in both x and y and the
    densities taken from their node interpolants.
    """
    gr, grw = np.asarray(gr, dtype=np.float64), np.asarray(grw, dtype=np.float64)
    nv, ng = gr.shape
    rho13 = np.asarray(rho13, dtype=np.float64).reshape(nv, ng)
    rho24 = np.asarray(rho24, dtype=np.float64).reshape(nv, ng)
    off = _disjoint_cells(rho13.ravel(), rho24.ravel(), gr.ravel(), grw.ravel(), k, ng)
    order = max(2 * ng, (k + ng + 1) // 2)
    nodes, x, wt, outer, inner = _triangle_rule(ng, order)
    h = grw.sum(axis=1)
    a = gr[:, 0] - h * (1 + nodes[0]) / 2
    r = a[:, None, None] + h[:, None, None] * x[None, :, None]
    s = a[:, None, None] + h[:, None, None] * x[None, :, None] * x[None, None, :]
    kj = (s / r) ** k / r * h[:, None, None] ** 2 * x[None, :, None]
    fo, go = rho13 @ outer.T, rho24 @ outer.T
    fi = np.einsum("cj,xyj->cxy", rho13, inner)
    gi = np.einsum("cj,xyj->cxy", rho24, inner)
    dens = fo[:, :, None] * gi + go[:, :, None] * fi
    diag = float(np.sum(dens * kj * wt[None, :, None] * wt[None, None, :]))
    return off + diag


# --------------------------------------------------------------------------
# Arbitrary-grid trapezoid Y^k (atomx src/atomx/numerics/quadrature.py)
# --------------------------------------------------------------------------
def coulomb_tables(r, k_max):
    """Block-scaled power tables (quadrature.py:190-231, ``_coulomb_tables``).

    Within a block x = r / r_anchor and (k_max + 1) log x <= 128, so the powers
    stay far from overflow; moving between blocks multiplies carried moments
    by (smaller anchor / larger anchor)^k <= 1.  Same numpy operations as the
    reference; returns (rk, inverse, cuts, transfers).
    """
    if isinstance(k_max, (bool, np.bool_)) or int(k_max) != k_max or k_max < 0:
        raise ValueError('Coulomb multipole rank must be a nonnegative integer')
    r = np.asarray(r, dtype=float)
    if (r.ndim != 1 or not r.size or not np.isfinite(r).all()
            or np.any(r <= 0) or np.any(np.diff(r) <= 0)):
        raise ValueError('Coulomb grid must be finite, positive and strictly increasing')
    logs, cuts = np.log(r), [0]
    span = 128. / (k_max + 1)
    while cuts[-1] < len(r):
        stop = int(np.searchsorted(logs, logs[cuts[-1]] + span, side='right'))
        cuts.append(max(cuts[-1] + 1, stop))
    cuts = np.asarray(cuts, dtype=np.int64)
    anchors = r[cuts[:-1]]
    rk = np.empty((k_max + 1, len(r)))
    inverse = np.empty_like(rk)
    orders = np.arange(k_max + 1)[:, None]
    for block in range(len(anchors)):
        lo, hi = cuts[block:block + 2]
        x = r[lo:hi] / anchors[block]
        rk[:, lo:hi] = x[None, :] ** orders
        inverse[:, lo:hi] = x[None, :] ** (-orders - 1) / anchors[block]
    transfers = ((anchors[:-1] / anchors[1:])[None, :] ** np.arange(k_max + 1)[:, None])
    return rk, inverse, cuts, transfers


def _grid_lib():
    lib = _lib()
    if not hasattr(lib, "_grid_bound"):
        lib.oracle_grid_yk_rho.argtypes = [_dptr, _dptr, ctypes.c_long, _dptr, _dptr, _lptr, ctypes.c_long, _dptr,
                                           ctypes.c_long, _dptr]
        lib.oracle_grid_yk_rho.restype = None
        lib.oracle_grid_pair_yk.argtypes = [_dptr, _dptr, _dptr, _dptr, _dptr, ctypes.c_long, _dptr, _dptr, _lptr,
                                            ctypes.c_long, _dptr, ctypes.c_long, _dptr]
        lib.oracle_grid_pair_yk.restype = None
        lib.oracle_grid_slater_rk.argtypes = [_dptr] * 9 + [ctypes.c_long, _dptr, _dptr, _lptr, ctypes.c_long,
                                                            _dptr, _dptr]
        lib.oracle_grid_slater_rk.restype = ctypes.c_double
        lib.oracle_grid_pair_dot_batch.argtypes = [_dptr, _dptr, _dptr, _dptr, ctypes.c_long, _lptr, _lptr, _lptr,
                                                   ctypes.POINTER(ctypes.c_ubyte), ctypes.c_long, _dptr,
                                                   ctypes.c_long, _lptr, _lptr, _dptr, ctypes.c_long, _dptr, _dptr,
                                                   _lptr, ctypes.c_long, _dptr, ctypes.c_long, ctypes.c_long, _dptr,
                                                   ctypes.c_int]
        lib.oracle_grid_pair_dot_batch.restype = None
        lib._grid_bound = True
    return lib


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def yk_on_grid(rho, r, k, i_cut=None):
    """quadrature.py:234-244: trapezoidal Green action on a radial density."""
    r = _c(r)
    rk, inverse, cuts, transfers = coulomb_tables(r, k)
    n = r.shape[0]
    ic = n - 1 if i_cut is None else min(int(i_cut), n - 1)
    y = np.empty(ic + 1 if ic + 1 > n else n)
    rk_k, inv_k, tr_k = _c(rk[k]), _c(inverse[k]), _c(transfers[k])
    _grid_lib().oracle_grid_yk_rho(_p(_c(rho)), _p(r), n, _p(rk_k), _p(inv_k), _p(_c(cuts, np.int64), _lptr),
                                   cuts.shape[0], _p(tr_k), ic, _p(y))
    return y[:ic + 1].copy()


def grid_slater_rk(P_a, Q_a, P_b, Q_b, P_c, Q_c, P_d, Q_d, r_grid, k):
    """quadrature.py:394-404: R^k(a,b,c,d) = Int rho_ac Y^k[rho_bd] dr."""
    r = _c(r_grid)
    rk, inverse, cuts, transfers = coulomb_tables(r, k)
    work = np.empty(r.shape[0])
    args = [_p(_c(x)) for x in (P_a, Q_a, P_b, Q_b, P_c, Q_c, P_d, Q_d)]
    return float(_grid_lib().oracle_grid_slater_rk(*args, _p(r), r.shape[0], _p(_c(rk[k])), _p(_c(inverse[k])),
                                                   _p(_c(cuts, np.int64), _lptr), cuts.shape[0],
                                                   _p(_c(transfers[k])), _p(work)))


def yk_pair_dot_batch_on_grid(PA, QA, PB, QB, rows_a, rows_b, rows_k, rows_ok, RhoA, cons_ptr, cons_rho, r,
                              i_cut=None, threads: int = 0):
    """quadrature.py:282-310: batched Int rho_w Y^k[rho_ab] dr with CSR consumers."""
    r = _c(r)
    n = r.shape[0]
    ic = n - 1 if i_cut is None else min(int(i_cut), n - 1)
    cons_ptr = _c(cons_ptr, np.int64)
    val = np.zeros(cons_ptr[-1] if cons_ptr.shape[0] else 0)
    rows_a = _c(rows_a, np.int64)
    if rows_a.shape[0] == 0:
        return val
    rows_k = _c(rows_k, np.int64)
    RK, inverse, cuts, transfers = coulomb_tables(r, int(rows_k.max()))
    PA, QA, PB, QB = (_c(x) for x in (PA, QA, PB, QB))
    RhoA = _c(RhoA)
    ok = _c(rows_ok, np.uint8)
    _grid_lib().oracle_grid_pair_dot_batch(
        _p(PA), _p(QA), _p(PB), _p(QB), PA.shape[1], _p(rows_a, _lptr), _p(_c(rows_b, np.int64), _lptr),
        _p(rows_k, _lptr), ok.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), rows_a.shape[0], _p(RhoA),
        RhoA.shape[1], _p(cons_ptr, _lptr), _p(_c(cons_rho, np.int64), _lptr), _p(r), n, _p(_c(RK)),
        _p(_c(inverse)), _p(_c(cuts, np.int64), _lptr), cuts.shape[0], _p(_c(transfers)), transfers.shape[1], ic,
        _p(val), threads)
    return val


def _potential_lib():
    lib = _lib()
    if not getattr(lib, "_potential_ready", False):
        lib.oracle_occupied_density.argtypes = [_dptr, _dptr, ctypes.c_long, ctypes.c_long, _dptr, ctypes.c_long,
                                                ctypes.c_long, _dptr]
        lib.oracle_occupied_density.restype = None
        lib.oracle_bspline_sym_matrix.argtypes = [_dptr, ctypes.c_int, _dptr, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, _dptr, ctypes.c_long, _dptr]
        lib.oracle_bspline_sym_matrix.restype = None
        lib._potential_ready = True
    return lib


def direct_potential_yk(bsp_data, ns, orbitals, target_kappa=None, target_idx=None):
    """(V_J_PP, V_J_QQ) <- src/atomx/methods/dirac_fock.py:931-967.

    Orbital values as evaluate.py:71-97 (``eval_P``/``eval_Q``), the density
    orbital by orbital in dict order (:939-952, C), Y^0 by ``yk_rows`` (C,
    yk.py:88-154), weights grw * Y^0 (:955) and the symmetrised matrices of
    ``_assemble_integral`` (numerics/bspline/integrals.py:18-56, C)."""
    lib = _potential_lib()
    nv, gr, grw = int(bsp_data["nv"]), np.asarray(bsp_data["gr"]), np.asarray(bsp_data["grw"])
    ng = gr.shape[1]
    n = nv * ng
    Ps, Qs, occ, target = [], [], [], -1
    for _kappa, orb_list in orbitals.items():
        for P, Q, o in orb_list:
            Ps.append(eval_P(P, bsp_data).ravel()), Qs.append(eval_Q(Q, bsp_data).ravel()), occ.append(float(o))
    if target_kappa is not None and target_idx is not None:
        lst = list(orbitals.get(target_kappa, []))
        if target_idx < len(lst):
            P, Q, _ = lst[target_idx]
            Ps.append(eval_P(P, bsp_data).ravel()), Qs.append(eval_Q(Q, bsp_data).ravel()), occ.append(0.0)
            target = len(Ps) - 1
    rho = np.zeros(n)
    if Ps:
        Pm, Qm = np.ascontiguousarray(Ps), np.ascontiguousarray(Qs)
        oc = np.ascontiguousarray(occ, dtype=np.float64)
        lib.oracle_occupied_density(_p(Pm), _p(Qm), n, Pm.shape[0], _p(oc), target, n, _p(rho))
    y = yk_rows(rho[None, :], 0, gr, grw, nv, ng)[0]
    weights = np.ascontiguousarray(grw.ravel() * y)
    out = []
    for key, kkey in (("bsp_p", "ksp"), ("bsp_q", "ksq")):
        b = np.ascontiguousarray(bsp_data[key], dtype=np.float64)
        ks = int(bsp_data[kkey])
        V = np.empty((int(ns), int(ns)))
        lib.oracle_bspline_sym_matrix(_p(b), ks, _p(b), ks, nv, ng, _p(weights), int(ns), _p(V))
        out.append(V)
    return out[0], out[1]


def compute_exchange_matrix(orb_b_P, orb_b_Q, bsp_data, k):
    """(K_PP, K_QQ) <- src/atomx/numerics/bspline/slater_yk.py:125-155 with the
    kernel :34-122 (C): orbital values as evaluate.py:71-97."""
    lib = _potential_lib()
    if not getattr(lib, "_exchange_ready", False):
        lib.oracle_exchange_matrix.argtypes = [_dptr, _dptr, _dptr, _dptr, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int, _dptr]
        lib.oracle_exchange_matrix.restype = None
        lib._exchange_ready = True
    nv, ns = int(bsp_data["nv"]), int(bsp_data["ns"])
    gr = np.ascontiguousarray(np.asarray(bsp_data["gr"]).ravel())
    grw = np.ascontiguousarray(np.asarray(bsp_data["grw"]).ravel())
    ng = np.asarray(bsp_data["gr"]).shape[1]
    out = []
    for coeffs, key, kkey, nkey in ((orb_b_P, "bsp_p", "ksp", "nsp"), (orb_b_Q, "bsp_q", "ksq", "nsq")):
        ks, nsb = int(bsp_data.get(kkey, bsp_data["ks"])), int(bsp_data.get(nkey, ns))
        bsp = np.ascontiguousarray(bsp_data.get(key, bsp_data["bsp_p"]), dtype=np.float64)
        fb = np.ascontiguousarray(eval_orbital_on_grid(coeffs, bsp, nv, ks, nsb).ravel())
        K = np.empty((nsb, nsb))
        lib.oracle_exchange_matrix(_p(fb), _p(bsp), _p(gr), _p(grw), nv, ng, ks, nsb, int(k), _p(K))
        out.append(K)
    return out[0], out[1]
