"""bench.py on the CPU: the reference arm's JSON line carries the keys the benchmark contract asks
for, and its runner times the reference CPU build or, without that build, the oracle's C
restatement of the Eulerian step."""
import contextlib
import io
import json
import os
import types

import pytest

import bench
from oracle import oracle as O


def test_reference_arm_line_has_the_contract_keys(monkeypatch):
    fake = {"gcell": 0.002, "psteps": 4.0e6, "ms_per_step": 2000.0, "wall_s": 12.0, "kind": "reference"}
    monkeypatch.setattr(bench, "run_reference", lambda workers, warm, steps: dict(fake, workers=workers))
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        bench.reference_arm(types.SimpleNamespace(warmup=3, steps=5), 1)
    line = json.loads(out.getvalue().strip().splitlines()[-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["steps"] == 5 and line["warmup"] == 3 and line["n_gpus"] == 1
    assert line["higher_is_better"] is True and line["value"] == fake["gcell"]
    assert line["e2e"] == {"value": fake["gcell"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"] and cb["cores"] >= 1 and cb["sample"]
    assert "extrapolated" in line["config"]["workload"]


@pytest.mark.parametrize("built", [True, False])
def test_reference_worker_times_the_build_or_the_port(monkeypatch, built):
    if built and not os.path.exists(O.REF_SO):
        pytest.skip("the reference CPU build is absent")
    if not built:
        monkeypatch.setattr(O, "REF_SO", os.path.join(os.path.dirname(O.REF_SO), "absent", "libgkm_ref.so"))
    assert bench._reference_built() == built
    steps = bench._ref_worker((12, 32, 7, 1, 2))
    assert len(steps) == 2
    for te, tp in steps:
        assert te > 0.0
        assert (tp > 0.0) if built else tp == 0.0
