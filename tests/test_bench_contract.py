"""bench.py's parts that need no GPU: the reference arm (the reference's own
score() on the host cores) prints the one JSON line the benchmark contract
asks for, with the GPU arm's workload keys, so the two lines compare the same
workload; and the roofline's stored traffic figures parse."""
from __future__ import annotations

import json
import subprocess
import sys

import pytest

import oracle as O
from conftest import ROOT

needs_ref = pytest.mark.skipif(not (O.REF_DIR / "libref_harness.so").exists(),
                               reason="needs the reference harness built into oracle/_ref")


@needs_ref
def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", "2",
                          "--steps", "1", "--warmup", "0", "--ref-seconds", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [x for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["unit"] == "GCUPS" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1 and d["value"] > 0
    n = d["config"]["n_sequences"]
    assert n == 20000 and d["config"]["pairs_per_gpu"] == n * (n - 1) // 2
    assert d["config"]["cells_per_gpu"] > 1e13 and d["config"]["workload"].startswith("config2")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_stored_traffic_figures_parse():
    """The roofline's DRAM traffic per launch comes from the committed ncu
    summary: read + write bytes of the full config-2 launch and the config-3
    launch (scaled from its 20,000-read capture)."""
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.measured_traffic("fast_all_pairs_kernel", "config2") == 68_590_000 + 777_680_000
    assert bench.measured_traffic("fast_all_pairs_kernel", "config3") == 1_711_140_000 + 19_383_600_000
    assert bench.measured_traffic("fast_all_pairs_kernel", "config9") is None
    gbs, src = bench.hbm_peak_gbs()
    assert gbs > 1000 and src.startswith("of ")
