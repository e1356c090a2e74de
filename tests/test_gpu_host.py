"""Tables delivered to pinned host memory with the copies overlapped
(``slater_rk_tables(..., host=True)``): bit-identical to the device tables of
the same engine, for both engines, including an ion whose cancelling table
the split engine recomputes in FP64."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(spec):
    from atomx_b200 import workloads as W
    from atomx_b200.tables import upload_ion
    return upload_ion(W.build_ion(spec))


@pytest.mark.parametrize("precision", ["fp64", "split"])
@pytest.mark.parametrize("which", ["neon_small", "batch42"])
def test_host_tables_equal_device_tables(precision, which):
    from atomx_b200 import workloads as W
    from atomx_b200.tables import tables_for
    spec = W.uneven_batch()[42] if which == "batch42" else getattr(W, which)()
    dev = _dev(spec)
    on_dev = tables_for(dev, precision)
    on_host = tables_for(dev, precision, host=True)
    assert not on_host.values.is_cuda and on_host.values.is_pinned()
    assert torch.equal(on_host.values, on_dev.values.cpu())
    for k in dev.plan.ks:
        assert torch.equal(on_host.table(k), on_dev.table(k).cpu())
    if precision == "split":
        assert on_host.info["fp64_multipoles"] == on_dev.info["fp64_multipoles"]
        if which == "batch42":
            assert 7 in on_host.info["fp64_multipoles"]


def test_slater_rk_tables_host_flag():
    from atomx_b200 import workloads as W
    from atomx_b200.tables import slater_rk_tables
    ion = W.build_ion(W.neon_small())
    a = slater_rk_tables(ion, precision="split", host=True)
    b = slater_rk_tables(ion, precision="split")
    assert torch.equal(a.values, b.values.cpu())
    assert np.isfinite(a.values.numpy()).all()


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_packed_host_tables_equal_device_tables(precision):
    """host=True, packed=True ships each table's upper triangle: it equals the
    device table's upper triangle bit for bit (same engine, same launches),
    and the expanded table equals the device table to rounding (diagonal
    tiles compute R(ac;bd) and R(bd;ac) separately; off-diagonal tiles are
    mirrored)."""
    import numpy as np
    import torch

    from atomx_b200 import workloads as W
    from atomx_b200.tables import HostPackedTables, slater_rk_tables
    ion = W.build_ion(W.neon_small())
    dev = slater_rk_tables(ion, precision=precision)
    host = slater_rk_tables(ion, precision=precision, host=True, packed=True)
    assert isinstance(host, HostPackedTables) and not host.values.is_cuda
    assert host.values.numel() == host.plan.unique_entries
    for k in dev.ks:
        d = dev.table(k).cpu().numpy()
        iu = np.triu_indices(d.shape[0])
        assert np.array_equal(host.packed(k), d[iu]), k
        assert np.max(np.abs(host.table(k) - d)) <= 1e-14 * np.abs(d).max(), k
    pr = dev.plan.pairs[dev.plan.pairs_of_k[1]]
    assert host.entry(1, tuple(pr[0]), tuple(pr[-1])) == dev.entry(1, tuple(pr[0]), tuple(pr[-1]))
    assert host.entry(1, tuple(pr[-1]), tuple(pr[0])) == dev.entry(1, tuple(pr[0]), tuple(pr[-1]))
    with pytest.raises(ValueError):
        slater_rk_tables(ion, precision=precision, packed=True)
    torch.cuda.synchronize()
