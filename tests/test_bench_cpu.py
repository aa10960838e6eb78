"""bench.py's reference arm on the CPU: its JSON line, and silence on the ranks other than 0.

The reference arm times the reference's FP64 kernel compiled for the host (or the NumPy oracle when
the captured kernels are absent) on a sample of the four-level workload; it needs no GPU.
"""

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", *args], cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=600)


def test_reference_arm_line_keeps_the_contract():
    sys.path.insert(0, str(ROOT))
    import bench
    r = _run({}, "--steps", "3", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["higher_is_better"] is True and d["steps"] == 3 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["config"] == bench.four_level_config(bench.SIDE, bench.NSTEPS, 1)
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] > 0 and cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    assert cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--gpus", "2", "--steps", "3", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
