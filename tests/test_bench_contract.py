"""The reference arm of bench.py on the CPU: its JSON line carries the keys
the bench contract names, and under several ranks only rank 0 works."""
from __future__ import annotations

import json
import os
import subprocess
import sys

from conftest import ROOT


def _run(extra_env=None, *args):
    env = dict(os.environ)
    env.update(extra_env or {})
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args]
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_line():
    p = _run({"WORLD_SIZE": "1", "RANK": "0"}, "--workload", "dam_break", "--steps", "2", "--warmup", "3")
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["metric"] == "particle-steps/s" and d["unit"] == "particle-steps/s"
    assert d["higher_is_better"] is True and d["steps"] == 2 and d["warmup"] == 3
    assert d["value"] > 0
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    # the GPU arm labels this workload the same way
    assert d["config"]["workload"] == "dam_break (16384 particles, 3 substep(s)/step, fp32)"


def test_reference_arm_other_ranks_do_nothing():
    p = _run({"WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"}, "--workload", "dam_break",
             "--steps", "2", "--warmup", "3")
    assert p.returncode == 0, p.stderr[-2000:]
    assert not [l for l in p.stdout.splitlines() if l.startswith("{")]


def test_issue_roofline_arithmetic():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    r = bench.issue_roofline("slab_1m", "fp32", "density", "list", 0.5, 2000.0, 100)
    # 100 SMs x 4 sub-partitions x 2e9 clocks = 8e11 warp instructions/s
    assert r["peak_warp_inst_per_s"] == 8e11
    assert r["frac"] == r["warp_instructions"] / 8e11 / 0.5e-3
    assert bench.issue_roofline("slab_1m", "fp32", "force", "list", 0.5, 2000.0, 100) is None
    assert bench.issue_roofline("slab_1m", "fp32", "density", "list", 0.5, None, 100) is None
