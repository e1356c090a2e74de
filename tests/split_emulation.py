"""CPU emulation of the split engine's two kernels (test helper).

``emulate_rows`` follows split_rows_kernel step by step on the packed factor
tables (same layout, same per-row power-of-two scaling, same residue rule);
``emulate_contract`` follows crt_syrk_kernel: exact int64 residue products
per modulus, the same reduction to [-128, 127], the same CRT constants and
FP64 recombination.  Tests compare the device buffers and tables with these.
"""
from __future__ import annotations

import numpy as np

from atomx_b200.split_plan import factor_table_layout


def unpack_table(flat, off, nv, ng):
    o = factor_table_layout(nv, ng)
    n = nv * ng
    t = flat[off:]
    nz = int(t[o["nz"]])
    z = t[o["z"]:o["z"] + nz * (ng + 1)].reshape(nz, ng + 1) if nz else np.zeros((0, ng + 1))
    return dict(u=t[:n].reshape(nv, ng), Lb=t[o["Lb"]:o["Lb"] + nv * ng * ng].reshape(nv, ng, ng),
                C=t[o["C"]:o["C"] + nv * ng].reshape(nv, ng), v0=t[o["v0"]:o["v0"] + ng],
                G00=t[o["G00"]:o["G00"] + ng * ng].reshape(ng, ng), sx=float(t[o["sx"]]),
                zcell=z[:, 0].astype(int), zvec=z[:, 1:])


def transform_rows(g, F, nv, ng):
    """[X | Z], left, right for rows g (rows, N) with one factor table F.

    left = [g_0, alpha sx, q / sx], right = [G_00 g_0, q / sx, alpha sx] with
    alpha = v_0 . g_0 and q = u_b . g_b (the suffix sum at cell 0)."""
    rows = g.shape[0]
    gb = g.reshape(rows, nv, ng)
    d = np.einsum("qmi,mi->qm", gb, F["u"])
    d[:, 0] = 0.0
    suf = np.cumsum(d[:, ::-1], axis=1)[:, ::-1]
    tn = np.concatenate([suf[:, 1:], np.zeros((rows, 1))], axis=1)
    g0 = gb[:, 0, :]
    alpha = g0 @ F["v0"]
    q = tn[:, 0]
    X = np.einsum("mij,qmi->qmj", F["Lb"], gb) + F["C"][None] * tn[:, :, None]
    X = X[:, 1:, :].reshape(rows, -1)
    Z = np.stack([gb[:, m, :] @ z for m, z in zip(F["zcell"], F["zvec"])], axis=1) if len(F["zcell"]) else \
        np.zeros((rows, 0))
    sx = F["sx"]
    left = np.concatenate([g0, (alpha * sx)[:, None], (q / sx)[:, None]], axis=1)
    right = np.concatenate([g0 @ F["G00"].T, (q / sx)[:, None], (alpha * sx)[:, None]], axis=1)
    return X, Z, left, right


def residues(xq, moduli):
    out = []
    for m in moduli:
        r = xq - m * np.rint(xq / m)
        r = np.where(r > 127, r - m, r)
        r = np.where(r < -128, r + m, r)
        out.append(r.astype(np.int64))
    return out


def merge_digits(res_list, moduli, pair_inv):
    """[0, m) residues -> merged digits exactly as the device merges them."""
    rs = [np.mod(np.asarray(r, dtype=np.int64), int(m)) for r, m in zip(res_list, moduli)]
    out = []
    for p in range(len(moduli) // 2):
        re, ro = rs[2 * p], rs[2 * p + 1]
        me, mo = int(moduli[2 * p]), int(moduli[2 * p + 1])
        t = np.mod((ro + 2 * mo - re) * int(pair_inv[p]), mo)
        out.append(re + me * t)
    if len(moduli) % 2:
        out.append(rs[-1])
    return out


def crt_value(res_list, moduli, f_hi, f_lo, M, pair_inv):
    digits = merge_digits(res_list, moduli, pair_inv)
    yh = np.zeros(digits[0].shape)
    yl = np.zeros(digits[0].shape)
    for d, fh, fl in zip(digits, f_hi, f_lo):
        yh = yh + d * fh
        yl = yl + d * fl
    return (yh - np.rint(yh)) * M + yl * M


def crt_exact(res_list, moduli):
    """Exact symmetric CRT with Python integers (|x| < M/2)."""
    ms = [int(m) for m in moduli]
    M = 1
    for m in ms:
        M *= m
    W = [(M // m) * pow((M // m) % m, -1, m) for m in ms]
    shape = res_list[0].shape
    flat = [np.asarray(r).ravel().tolist() for r in res_list]
    out = np.empty(len(flat[0]), dtype=np.float64)
    for idx in range(len(flat[0])):
        x = sum(int(flat[i][idx]) * W[i] for i in range(len(ms))) % M
        if x > M // 2:
            x -= M
        out[idx] = float(x)
    return out.reshape(shape)


def reduce_mod(v, m):
    r = v - m * np.rint(v / m).astype(np.int64)
    for _ in range(2):
        r = np.where(r < -128, r + m, r)
        r = np.where(r > 127, r - m, r)
    return r


def emulate_table(Ares, Bres, rowscale, left, right, moduli, f_hi, f_lo, M, pair_inv):
    """One symmetric table from residue rows (lists per modulus of (n, K))."""
    res = []
    for a, b, m in zip(Ares, Bres, moduli):
        res.append(reduce_mod(a.astype(np.int64) @ b.astype(np.int64).T, int(m)))
    x = crt_value(res, moduli, f_hi, f_lo, M, pair_inv)
    return x * np.outer(rowscale, rowscale) + left @ right.T
