"""bench.py's reference arm on the host (no GPU needed): the JSON line keeps
the contract's keys, and ranks other than 0 exit quietly."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CMD = [sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"]


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run(CMD, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    # one step is slice 0 of 4: every 4th bd row of each multipole table
    # against all of its ac rows, measured (nothing extrapolated)
    from atomx_b200 import plan as PL
    from atomx_b200 import workloads as W
    spec = W.ytterbium_scaleup()
    plan = PL.make_plan(W.build_ion(spec).kappa, spec.k_max)
    assert plan.ordered_entries == 318112753
    want = sum(((plan.n_of_k(k) + 3) // 4) * plan.n_of_k(k) for k in plan.ks)
    assert line["config"]["entries_per_step"] == want
    assert abs(line["ms_per_step"] - line["cpu_baseline"]["seconds_measured"] * 1e3) < 20.0


def test_reference_slices_cover_the_table_once():
    import numpy as np

    from atomx_b200 import plan as PL
    from bench import REFERENCE_SLICES
    plan = PL.make_plan(np.array([-1, -1, 1, -2, -2, 2, -3]), 4)
    for k in plan.ks:
        nk = plan.n_of_k(k)
        seen = np.concatenate([np.arange(p, nk, REFERENCE_SLICES) for p in range(REFERENCE_SLICES)])
        assert np.array_equal(np.sort(seen), np.arange(nk))


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1")
    out = subprocess.run(CMD, cwd=ROOT, capture_output=True, text=True, timeout=120, env=env)
    assert out.returncode == 0 and out.stdout.strip() == ""
