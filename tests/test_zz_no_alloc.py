"""rkb_split_rows_noalloc against rkb_split_rows, through the C ABI.

The no-alloc variant exists for hosts that cannot call cudaMalloc on this
path (a C or Fortran program that links only the ABI and owns a device pool,
or a process that plans all device memory up front): its FP64 row workspace
is a fixed array inside the library instead of a caller buffer.  Two calls in
a row, with different ions, row ranges and widths, must give the same
residues, scales, correction vectors and bounds as the entry point that takes
a caller workspace; a request larger than the fixed array is refused.

This file sorts last so that a run stopping at the first failure has run
every other test before it.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

#: RKB_SPLIT_ROWS_NOALLOC_MAX_DOUBLES in include/rkb200.h (16 MiB of doubles)
CAP = 2 * 1024 * 1024
#: doubles per row of the row record (d_cbound)
CB_STRIDE = 8


def _outputs(torch, eng, nr):
    d = eng.ktab.device
    res_a = torch.zeros((eng.n_mod, nr, eng.kpad), dtype=torch.int8, device=d)
    res_b = torch.zeros_like(res_a) if eng.resB is not None else None
    return dict(resA=res_a, resB=res_b, rowscale=torch.empty(nr, dtype=torch.float64, device=d),
                left=torch.empty((nr, eng.cwp), dtype=torch.float64, device=d),
                right=torch.empty((nr, eng.cwp), dtype=torch.float64, device=d),
                cbound=torch.empty((nr, CB_STRIDE), dtype=torch.float64, device=d))


def _call(torch, eng, r0, nr, noalloc, row_base=0):
    """Rows [r0, r0 + nr) of eng's plan into fresh output buffers.

    The rows land at output rows [row_base, row_base + nr); the entry points
    index their workspace the same way, so a caller workspace of
    (row_base + nr) rows is what rkb_split_rows needs.  Only the written rows
    are returned.
    """
    from atomx_b200 import _native
    L = _native.load()
    dev = eng.dev
    total = row_base + nr
    out = _outputs(torch, eng, total)
    head = (dev.Pv.data_ptr(), dev.Qv.data_ptr(), dev.n, dev.pairs.data_ptr(),
            dev.row_pair.data_ptr() + 8 * r0, dev.row_k.data_ptr() + 4 * r0, nr, dev.w.data_ptr(), dev.nv,
            dev.ng, eng.ktab.data_ptr(), eng.koff.data_ptr(), eng.bits, eng.n_mod, eng._mod_c[0],
            out["resA"].data_ptr(), _native.ptr(out["resB"]), eng.kpad, row_base, total,
            out["rowscale"].data_ptr(), out["left"].data_ptr(), out["right"].data_ptr(),
            out["cbound"].data_ptr(), eng.cwp)
    if noalloc:
        st = L.rkb_split_rows_noalloc(*head, eng.zcount.data_ptr(), None)
    else:
        xwork = torch.empty((total, eng.kpad), dtype=torch.float64, device=eng.ktab.device)
        st = L.rkb_split_rows(*head, xwork.data_ptr(), eng.zcount.data_ptr(), None)
    _native.check(st, "rkb_split_rows_noalloc" if noalloc else "rkb_split_rows")
    torch.cuda.synchronize()
    sl = slice(row_base, total)
    return {key: (None if v is None else (v[:, sl] if key in ("resA", "resB") else v[sl]))
            for key, v in out.items()}


def _same(a, b):
    """Bit-identical outputs: both calls run the same kernels on the same rows."""
    import torch
    for key in a:
        if a[key] is None:
            assert b[key] is None, key
        elif a[key].dtype == torch.int8:
            assert torch.equal(a[key], b[key]), key
        else:
            assert torch.allclose(a[key], b[key], rtol=0.0, atol=0.0, equal_nan=True), key


def test_noalloc_rows_match_caller_workspace_twice():
    import torch

    from atomx_b200 import _native
    from atomx_b200 import tables as T
    from atomx_b200 import workloads as W
    from atomx_b200.split import SplitEngine
    _native.require_device()

    # first call: every row of the Z=10 table
    neon = SplitEngine(T.upload_ion(W.build_ion(W.neon_small())))
    n1 = neon.dev.plan.n_rows
    ref1 = _call(torch, neon, 0, n1, noalloc=False)
    got1 = _call(torch, neon, 0, n1, noalloc=True)
    _same(ref1, got1)
    assert np.all(np.isfinite(got1["rowscale"].cpu().numpy()))

    # second call: a different ion, row width and row range (Z=70, N=896)
    yb = SplitEngine(T.upload_ion(W.build_ion(W.ytterbium_scaleup())))
    r0, nr = 5000, CAP // yb.kpad
    ref2 = _call(torch, yb, r0, nr, noalloc=False)
    got2 = _call(torch, yb, r0, nr, noalloc=True)
    _same(ref2, got2)
    assert bool((got2["resA"] != 0).any())

    # the first ion again: the workspace still holds the second call's rows
    got3 = _call(torch, neon, 0, n1, noalloc=True)
    _same(ref1, got3)

    # rows placed at an offset: row_base + nrows is exactly the capacity, so
    # the last row ends on the last double of the fixed workspace
    base = 700
    nb = CAP // yb.kpad - base
    ref4 = _call(torch, yb, 1234, nb, noalloc=False, row_base=base)
    got4 = _call(torch, yb, 1234, nb, noalloc=True, row_base=base)
    _same(ref4, got4)
    assert bool((got4["resA"] != 0).any())

    # a request beyond the fixed workspace is refused before any launch,
    # whether the rows alone or the offset plus the rows overflow it
    with pytest.raises(ValueError, match="fixed workspace"):
        _call(torch, yb, 0, nr + 1, noalloc=True)
    with pytest.raises(ValueError, match="fixed workspace"):
        _call(torch, yb, 0, nb + 1, noalloc=True, row_base=base)
    with pytest.raises(ValueError, match="fixed workspace"):
        _call(torch, yb, 0, 1, noalloc=True, row_base=CAP // yb.kpad)
