"""Streamed tables: per-multipole tables handed to a caller sink.

The Z=54 CI-scale table (N=2112, 300 spinors, k <= 16, 1.95e9 entries) is
streamed through the split engine without ever holding the whole table on
the device. Every streamed table must equal the materialised run bit for bit:
each tile is computed by the same kernel with the same inputs. Size-free
properties check this at full size: per-k sums and sums of squares, and
sampled kappa-block tiles.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


class _Collect:
    """Sink keeping a device copy of every table (small cases only)."""

    def __init__(self):
        self.tables = {}

    def __call__(self, k, table, blocks, stream):
        with torch.cuda.stream(stream):
            self.tables[k] = table.clone()
        self.blocks = getattr(self, "blocks", {})
        self.blocks[k] = blocks


def _bit_checksums(table):
    """Order-free checksums of the bit patterns (integer sums wrap mod 2^64)."""
    bits = table.contiguous().view(torch.int64)
    return bits.sum(), ((bits >> 20) * (bits & 0xFFFFF)).sum()


class _Checksums:
    """Sink recording per-k checksums and a few kappa-block tiles."""

    def __init__(self, picks):
        self.sums, self.tiles, self.picks = {}, {}, picks

    def __call__(self, k, table, blocks, stream):
        from atomx_b200.tables import iter_blocks
        with torch.cuda.stream(stream):
            self.sums[k] = (*_bit_checksums(table), torch.isfinite(table).all())
            for b1, b2, tile in iter_blocks(table, blocks):
                if (k, b1, b2) in self.picks:
                    self.tiles[(k, b1, b2)] = tile.clone()


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_stream_neon_equals_materialised(precision):
    from atomx_b200 import workloads as W
    from atomx_b200.tables import iter_blocks, slater_rk_tables
    ion = W.build_ion(W.neon_small())
    full = slater_rk_tables(ion, precision=precision)
    sink = _Collect()
    summary = slater_rk_tables(ion, precision=precision, sink=sink)
    torch.cuda.synchronize()
    assert sorted(sink.tables) == sorted(full.ks) == sorted(summary.ks)
    for k in full.ks:
        assert torch.equal(sink.tables[k], full.table(k)), k
        # the kappa blocks tile the table exactly
        covered = sum(t.numel() for _, _, t in iter_blocks(sink.tables[k], sink.blocks[k]))
        assert covered == sink.tables[k].numel()


def test_host_sink_ytterbium_k2():
    from atomx_b200 import workloads as W
    from atomx_b200.tables import HostTableSink, slater_rk_tables
    ion = W.build_ion(W.ytterbium_scaleup())
    full = slater_rk_tables(ion, k_max=2, precision="split")
    sink = HostTableSink()
    slater_rk_tables(ion, k_max=2, precision="split", sink=sink)
    host = sink.wait()
    for k in full.ks:
        np.testing.assert_array_equal(host[k].numpy(), full.table(k).cpu().numpy())


def test_stream_xenon_ci_table_never_materialised():
    from atomx_b200 import workloads as W
    from atomx_b200.tables import slater_rk_tables
    ion = W.build_ion(W.xenon_ci_table())
    picks = {(0, 0, 0), (1, 2, 36), (8, 46, 15), (16, 170, 164)}
    sink = _Checksums(picks)
    summary = slater_rk_tables(ion, precision="split", sink=sink)
    torch.cuda.synchronize()
    plan = summary.plan
    table_bytes = 8 * plan.ordered_entries
    assert plan.ordered_entries > 1.9e9
    assert all(bool(v[2]) for v in sink.sums.values())
    streamed = {k: (int(a), int(b)) for k, (a, b, _) in sink.sums.items()}
    tiles = {key: t.cpu() for key, t in sink.tiles.items()}
    del sink
    torch.cuda.empty_cache()
    full = slater_rk_tables(ion, precision="split")
    # the streamed run holds its rows and two rotating multipole buffers (the
    # largest table is 14 524^2 entries), never the 15.6 GB table
    nmax = max(plan.n_of_k(k) for k in plan.ks)
    assert summary.device_bytes < table_bytes, (summary.device_bytes, table_bytes)
    assert summary.device_bytes < full.info["device_bytes"] - table_bytes + 2 * 8 * nmax * nmax + 1
    for k in full.ks:
        t = full.table(k)
        assert streamed[k] == tuple(int(c) for c in _bit_checksums(t)), k
    from atomx_b200.tables import iter_blocks
    for k in {key[0] for key in picks}:
        for b1, b2, tile in iter_blocks(full.table(k), plan.block_ranges_of_k(k)):
            if (k, b1, b2) in tiles:
                assert torch.equal(tiles[(k, b1, b2)], tile.cpu()), (k, b1, b2)
    assert len(tiles) == len(picks)
