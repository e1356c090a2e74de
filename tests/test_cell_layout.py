"""Host check of the cell engine's block-matrix form (no GPU): with the
oracle's banks laid out as K_full[(ip, i)][(jp, j)] (component blocks padded
to 16 columns) and the banded pair densities in the same order, the bilinear
form D(ab) K_full D(cd)^T reproduces the oracle's cell integral (atomx's
full-bank path, bit-pinned to atomx), and W = D K_full^T rows hold the
banded case-1 potentials."""
import numpy as np
import pytest

from oracle import cell as OC


def _round16(x):
    return (x + 15) // 16 * 16


def _kfull(bd, k, banks):
    ns, ksp, ksq = bd["ns"], bd["ksp"], bd["ksq"]
    kp, kq = _round16(ksp * ns), _round16(ksq * ns)
    K = np.zeros((kp + kq, kp + kq))
    off = {"p": 0, "q": kp}
    ks = {"p": ksp, "q": ksq}
    for itype in OC.ITYPES:
        left, right = itype[0], itype[1]
        rkb = banks(k, itype)  # (ns, ns, ks_l, ks_r)
        blk = rkb.transpose(2, 0, 3, 1).reshape(ks[left] * ns, ks[right] * ns)
        K[off[left]:off[left] + ks[left] * ns, off[right]:off[right] + ks[right] * ns] = blk
    return K, kp


def _drow(bd, kp, Pa, Qa, Pb, Qb):
    ns = bd["ns"]
    d = np.zeros(kp + _round16(bd["ksq"] * ns))
    dp = OC.density_sym(Pa, Pb, bd["nsp"], bd["ksp"])
    dq = OC.density_sym(Qa, Qb, bd["nsq"], bd["ksq"])
    for off, dens, ks in ((0, dp, bd["ksp"]), (kp, dq, bd["ksq"])):
        full = np.zeros((ns, ks))
        full[:dens.shape[0]] = dens
        d[off:off + ks * ns] = full.T.reshape(-1)
    return d


@pytest.mark.parametrize("k", [0, 1, 2])
def test_bilinear_form_equals_cell_integral(k):
    from atomx_b200 import workloads as W
    ion = W.build_ion(W.neon_small())
    bd = ion.bsp
    banks = OC.Banks(bd)
    K, kp = _kfull(bd, k, banks)
    rng = np.random.default_rng(k)
    for _ in range(6):
        a, b, c, d = rng.integers(0, 4, 4)
        ref = OC.slater_rk_cell(ion.P[a], ion.Q[a], ion.P[b], ion.Q[b], ion.P[c], ion.Q[c], ion.P[d], ion.Q[d], bd,
                                k, banks)
        dl = _drow(bd, kp, ion.P[a], ion.Q[a], ion.P[b], ion.Q[b])
        dr = _drow(bd, kp, ion.P[c], ion.Q[c], ion.P[d], ion.Q[d])
        assert dl @ K @ dr == pytest.approx(ref, rel=1e-13, abs=1e-15)


def test_potential_rows_are_case1_bands():
    from atomx_b200 import workloads as W
    ion = W.build_ion(W.neon_small())
    bd = ion.bsp
    banks = OC.Banks(bd)
    K, kp = _kfull(bd, 1, banks)
    ns = bd["ns"]
    P, Q = ion.P[1], ion.Q[1]
    row = np.zeros(K.shape[0])
    dp, dq = OC.density_sym(P, P, ns, bd["ksp"]), OC.density_sym(Q, Q, ns, bd["ksq"])
    row[:bd["ksp"] * ns] = dp.T.reshape(-1)
    row[kp:kp + bd["ksq"] * ns] = dq.T.reshape(-1)
    w = K @ row
    vp = OC.convol_case1(banks(1, "pppp"), dp, ns, bd["ksp"], bd["ksp"]) + \
        OC.convol_case1(banks(1, "pqpq"), dq, ns, bd["ksp"], bd["ksq"])
    assert np.allclose(w[:bd["ksp"] * ns].reshape(bd["ksp"], ns).T, vp, rtol=0, atol=1e-14 * np.abs(vp).max())
