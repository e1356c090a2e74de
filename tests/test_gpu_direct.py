"""Potential matrices on the device against atomx's outputs and the oracle:
the direct (Hartree) potential (DFSolver._build_direct_potential_yk, atomx
methods/dirac_fock.py:931-967) and the exchange matrices
(compute_exchange_matrix, numerics/bspline/slater_yk.py:125).

The device evaluates the orbitals with its own reduction order, so the
density and Y^0 differ from atomx's in the last bits; the matrices are
compared within 1e-13 of each matrix's largest entry, the gate of the Y^k
rows themselves.  The density kernel and the matrix kernel alone are also
checked against the oracle on identical device inputs, bit for bit.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle
from test_oracle_direct import _case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = 1e-13


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(GOLDEN, "direct_potential.npz"))


def _close(got, ref, tol=TOL):
    scale = np.abs(ref).max()
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= tol * scale, np.abs(got - ref).max() / scale


@pytest.mark.parametrize("name", ["neon", "batch5"])
def test_direct_potential_matches_atomx(g, name):
    from atomx_b200.dirac_fock import build_direct_potential_yk
    bd, orbitals, (tk, ti) = _case(g, name)
    vpp, vqq = build_direct_potential_yk(bd, bd["ns"], orbitals)
    _close(vpp, g[f"{name}_VPP"])
    _close(vqq, g[f"{name}_VQQ"])
    assert np.array_equal(vpp, vpp.T) and np.array_equal(vqq, vqq.T)
    vpp_t, vqq_t = build_direct_potential_yk(bd, bd["ns"], orbitals, tk, ti)
    _close(vpp_t, g[f"{name}_VPP_t"])
    _close(vqq_t, g[f"{name}_VQQ_t"])


def test_method_form_reads_solver_attributes(g):
    from types import SimpleNamespace

    from atomx_b200.dirac_fock import direct_potential_yk_method
    bd, orbitals, _ = _case(g, "neon")
    me = SimpleNamespace(bsp_data=bd, ns=bd["ns"], ks=bd["ks"])
    vpp, vqq = direct_potential_yk_method(me, orbitals)
    _close(vpp, g["neon_VPP"])


def test_kernels_equal_oracle_on_same_inputs(g):
    """Density and matrix kernels alone, fed the oracle's own orbital values
    and Y^0: every operation is in the oracle's order, so bit for bit."""
    from atomx_b200 import _native
    L = _native.load()
    bd, orbitals, (tk, ti) = _case(g, "batch5")
    nv, ng = bd["gr"].shape
    n = nv * ng
    Pv = np.array([oracle.eval_P(P, bd).ravel() for lst in orbitals.values() for P, _, _ in lst])
    Qv = np.array([oracle.eval_Q(Q, bd).ravel() for lst in orbitals.values() for _, Q, _ in lst])
    occ = np.array([o for lst in orbitals.values() for _, _, o in lst])
    ref = np.zeros(n)
    lib = oracle._potential_lib()
    P_, Q_, o_ = (np.ascontiguousarray(x) for x in (Pv, Qv, occ))
    lib.oracle_occupied_density(oracle._p(P_), oracle._p(Q_), n, P_.shape[0], oracle._p(o_), 3, n, oracle._p(ref))
    dP, dQ, dO = (torch.as_tensor(x, device="cuda") for x in (P_, Q_, o_))
    rho = torch.empty(n, dtype=torch.float64, device="cuda")
    _native.check(L.rkb_occupied_density(dP.data_ptr(), dQ.data_ptr(), n, P_.shape[0], dO.data_ptr(), 3, n,
                                         rho.data_ptr(), None), "rkb_occupied_density")
    np.testing.assert_array_equal(rho.cpu().numpy(), ref)
    y = oracle.yk_rows(ref[None, :], 0, bd["gr"], bd["grw"], nv, ng)[0]
    weights = np.ascontiguousarray(bd["grw"].ravel() * y)
    b = np.ascontiguousarray(bd["bsp_p"])
    ns = bd["ns"]
    V = np.empty((ns, ns))
    lib.oracle_bspline_sym_matrix(oracle._p(b), bd["ksp"], oracle._p(b), bd["ksp"], nv, ng, oracle._p(weights), ns,
                                  oracle._p(V))
    dB, dW, dY = (torch.as_tensor(x, device="cuda") for x in (b, np.ascontiguousarray(bd["grw"].ravel()), y))
    out = torch.empty((ns, ns), dtype=torch.float64, device="cuda")
    _native.check(L.rkb_bspline_sym_matrix(dB.data_ptr(), bd["ksp"], dB.data_ptr(), bd["ksp"], nv, ng, dW.data_ptr(),
                                           dY.data_ptr(), ns, out.data_ptr(), None), "rkb_bspline_sym_matrix")
    np.testing.assert_array_equal(out.cpu().numpy(), V)


def test_errors():
    from atomx_b200 import _native
    L = _native.load()
    with pytest.raises(ValueError):
        _native.check(L.rkb_occupied_density(0, 0, 10, 2, 0, 5, 10, 0, None), "rkb_occupied_density")


# ------------------------------------------------------------------ exchange
@pytest.fixture(scope="module")
def gx():
    return np.load(os.path.join(GOLDEN, "exchange_matrix.npz"))


@pytest.mark.parametrize("name", ["neon", "batch5"])
def test_exchange_matrix_matches_atomx(gx, name):
    from test_oracle_exchange import exchange_case

    from atomx_b200.slater_yk import compute_exchange_matrix
    bd, picks = exchange_case(gx, name)
    for orb, k in picks:
        kpp, kqq = compute_exchange_matrix(gx[f"{name}_P{orb}"], gx[f"{name}_Q{orb}"], bd, k)
        _close(kpp, gx[f"{name}_KPP_{orb}_{k}"])
        _close(kqq, gx[f"{name}_KQQ_{orb}_{k}"])


def test_exchange_kernel_equals_oracle_on_same_orbital(gx):
    """Fed the oracle's own orbital values, the kernel runs every sum in the
    reference's order: bit for bit."""
    from test_oracle_exchange import exchange_case

    from atomx_b200 import _native
    L = _native.load()
    bd, picks = exchange_case(gx, "batch5")
    nv, ng = bd["gr"].shape
    lib = oracle._potential_lib()
    oracle.compute_exchange_matrix(gx["batch5_P0"], gx["batch5_Q0"], bd, 0)  # sets the C signatures
    r = np.ascontiguousarray(bd["gr"].ravel())
    w = np.ascontiguousarray(bd["grw"].ravel())
    for orb, k in picks:
        fb = np.ascontiguousarray(oracle.eval_P(gx[f"batch5_P{orb}"], bd).ravel())
        b = np.ascontiguousarray(bd["bsp_p"])
        ns = bd["nsp"]
        ref = np.empty((ns, ns))
        lib.oracle_exchange_matrix(oracle._p(fb), oracle._p(b), oracle._p(r), oracle._p(w), nv, ng, bd["ksp"], ns, k,
                                   oracle._p(ref))
        dfb, db, dr, dw = (torch.as_tensor(x, device="cuda") for x in (fb, b, r, w))
        K = torch.empty((ns, ns), dtype=torch.float64, device="cuda")
        _native.check(L.rkb_exchange_matrix(dfb.data_ptr(), db.data_ptr(), dr.data_ptr(), dw.data_ptr(), nv, ng,
                                            bd["ksp"], ns, k, K.data_ptr(), None), "rkb_exchange_matrix")
        np.testing.assert_array_equal(K.cpu().numpy(), ref)


def test_exchange_errors(gx):
    from test_oracle_exchange import exchange_case

    from atomx_b200.slater_yk import compute_exchange_matrix
    bd, _ = exchange_case(gx, "neon")
    with pytest.raises(ValueError):
        compute_exchange_matrix(gx["neon_P0"], gx["neon_Q0"], bd, -1)
    with pytest.raises(ValueError):
        compute_exchange_matrix(gx["neon_P0"], gx["neon_Q0"], bd, 1.5)
