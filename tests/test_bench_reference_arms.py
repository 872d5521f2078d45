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


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
def test_histogram_reference_arm_same_config_and_no_library_of_ours():
    """The headline's reference arm (histogram workload, here on an 8^3-cell cube): the seed-0 workload
    and the config dict of our arm; only the reference's own build is mapped (neither our CUDA library
    nor the oracle port); the histogram hash is the one of the oracle's histogram of the same cube."""
    code = ("import runpy, sys\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--cells', '8', '--steps', '1', '--warmup', '0']\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\nexcept SystemExit:\n    pass\n"
            "print('MAPS ' + ' '.join(sorted({l.split()[-1] for l in open('/proc/self/maps') if l.rstrip().endswith('.so')})))\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][0])
    maps = [l for l in r.stdout.splitlines() if l.startswith("MAPS ")][0].split()[1:]
    assert any(m.endswith("oracle/_ref/libxnsref.so") for m in maps)
    assert not any(m.endswith("libxns_b200.so") or m.endswith("liboracle.so") for m in maps), maps
    sys.path.insert(0, ROOT)
    import bench
    els, nh = bench.workload(0, 8)[:2]
    assert d["config"] == bench.config_block(els, nh, 8)
    from oracle import Oracle
    assert d["histogram_sha256"] == bench.hist_sha256(Oracle().hist(els, nh, bench.BIN))
