"""CPU: bench.py --impl reference for every workload prints one JSON line with the contract's keys and
the metric and unit of our arm for that workload (small sizes where the workload takes them)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

HAVE_REF = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libxnsref.so"))

# (workload, extra arguments, metric, unit) -- the metric and unit of our arm for the workload
ARMS = [("debye", [], "atom-pairs/s", "pairs/s"),
        ("2d", ["--cells2d", "6", "--mesh2d", "32"], "terms/s", "(atom, q-point) terms/s"),
        ("batch", [], "patterns/s", "patterns/s"),
        ("build", [], "site pairs/s (structure build)", "pairs/s")]


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("workload,extra,metric,unit", ARMS)
def test_reference_arm(workload, extra, metric, unit):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", workload,
                        "--steps", "1", "--warmup", "0"] + extra, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == metric and d["unit"] == unit
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "reference"
    assert d["e2e"] == {"value": d["value"], "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    for k in ("n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "vs_baseline", "dtype", "data",
              "config"):
        assert k in d
