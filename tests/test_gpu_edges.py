"""Edge cases of the table engines: the smallest tables, non-finite inputs,
grids beyond the split engine's contraction limit, one-ion batches and
one-table streams.  Values are checked against the oracle (the reference
algorithm) on inputs generated on the test host."""
import numpy as np
import pytest

from oracle import oracle
from oracle_entries import sampled_oracle_entries

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _ion(shells, k_max, ns=40, ks=7, ng=7, Z=10.0, seed=None):
    from atomx_b200 import workloads as W
    spec = W.IonSpec(Z=Z, ns=ns, ks=ks, n_gauss=ng, r_min=1e-5, r_max=40.0, shells=shells, k_max=k_max, seed=seed,
                     name="edge")
    ion = W.build_ion(spec)
    bd = ion.bsp
    Pg = np.array([oracle.eval_P(c, bd).ravel() for c in ion.P])
    Qg = np.array([oracle.eval_Q(c, bd).ravel() for c in ion.Q])
    return spec, ion, Pg, Qg


def _check_vs_oracle(tab, ion, Pg, Qg, gate):
    for k, ii, jj, ref in sampled_oracle_entries(ion, Pg, Qg, tab.plan, per_k=8, seed=3):
        T = tab.table(k).cpu().numpy()
        d = np.abs(np.diag(T))
        err = np.abs(T[ii, jj] - ref) / np.sqrt(d[ii] * d[jj])
        assert err.max() <= gate, (k, err.max())


@pytest.mark.parametrize("precision,gate", [("fp64", 1e-13), ("split", 1e-10)])
def test_single_spinor_one_by_one_table(precision, gate):
    from atomx_b200.tables import slater_rk_tables_from_values
    spec, ion, Pg, Qg = _ion(((-1, 1),), k_max=0)
    tab = slater_rk_tables_from_values(Pg, Qg, ion.kappa, ion.bsp["gr"], ion.bsp["grw"], 0, precision=precision)
    assert tab.ks == [0] and tab.table(0).shape == (1, 1)
    _check_vs_oracle(tab, ion, Pg, Qg, gate)


@pytest.mark.parametrize("precision,gate", [("fp64", 1e-13), ("split", 1e-10)])
def test_k_max_zero_and_ragged_blocks(precision, gate):
    from atomx_b200.tables import slater_rk_tables_from_values
    spec, ion, Pg, Qg = _ion(((-1, 3), (1, 2), (-2, 5)), k_max=0, seed=7)
    tab = slater_rk_tables_from_values(Pg, Qg, ion.kappa, ion.bsp["gr"], ion.bsp["grw"], 0, precision=precision)
    assert tab.ks == [0]
    _check_vs_oracle(tab, ion, Pg, Qg, gate)


def test_non_finite_orbital_values():
    """A NaN in an orbital: the split engine reports it (FloatingPointError,
    atomx's exception for non-finite integrals); the FP64 engine returns NaN in
    exactly the entries that involve that orbital, as slater_rk_poisson does."""
    from atomx_b200.tables import slater_rk_tables_from_values
    spec, ion, Pg, Qg = _ion(((-1, 2), (1, 1), (-2, 1)), k_max=2)
    Pg = Pg.copy()
    Pg[1, 57] = np.nan
    bd = ion.bsp
    with pytest.raises(FloatingPointError):
        slater_rk_tables_from_values(Pg, Qg, ion.kappa, bd["gr"], bd["grw"], 2, precision="split")
    tab = slater_rk_tables_from_values(Pg, Qg, ion.kappa, bd["gr"], bd["grw"], 2, precision="fp64")
    plan = tab.plan
    for k in tab.ks:
        T = tab.table(k).cpu().numpy()
        touched = np.array([1 in plan.pairs[p] for p in plan.pairs_of_k[k]])
        bad = np.isnan(T)
        assert np.array_equal(bad, touched[:, None] | touched[None, :]), k


def test_grid_beyond_split_limit_is_refused_before_launch():
    from atomx_b200.tables import slater_rk_tables_from_values
    spec, ion, Pg, Qg = _ion(((-1, 2),), k_max=0, ns=420, ks=9, ng=9)
    bd = ion.bsp
    with pytest.raises(ValueError, match="too long for the split engine"):
        slater_rk_tables_from_values(Pg, Qg, ion.kappa, bd["gr"], bd["grw"], 0, precision="split")
    tab = slater_rk_tables_from_values(Pg, Qg, ion.kappa, bd["gr"], bd["grw"], 0, precision="fp64")
    _check_vs_oracle(tab, ion, Pg, Qg, 1e-13)


def test_one_ion_batch_and_one_table_stream():
    from atomx_b200.batch import SplitBatch
    from atomx_b200.tables import slater_rk_tables_from_values, stream_tables, upload_values
    spec, ion, Pg, Qg = _ion(((-1, 1),), k_max=0)
    bd = ion.bsp
    dev = upload_values(Pg, Qg, ion.kappa, bd["gr"], bd["grw"], 0)
    b = SplitBatch([dev])
    b.replay()
    torch.cuda.synchronize()
    b.check_status()
    single = slater_rk_tables_from_values(Pg, Qg, ion.kappa, bd["gr"], bd["grw"], 0, precision="split")
    assert torch.equal(b.table(0, 0), single.table(0))
    got = {}
    stream_tables(dev, lambda k, t, blocks, s: got.__setitem__(k, t.clone()), precision="split")
    torch.cuda.synchronize()
    assert list(got) == [0] and torch.equal(got[0], single.table(0))


def test_empty_ion_is_a_value_error():
    from atomx_b200.plan import make_plan
    with pytest.raises(ValueError):
        make_plan([], 2)
    with pytest.raises(ValueError):
        make_plan([-1], -1)
