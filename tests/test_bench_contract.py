"""bench.py's reference arm runs on the CPU alone: one JSON line with the
metric, unit and config of the B200 arm, a cpu_baseline describing the run, and
an e2e entry with no host-device traffic."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "fluid4k", "--steps", "2", "--warmup", "3"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "atom-steps/s" and d["unit"] == "atom-steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] >= 1 and d["n_gpus"] == 1
    assert d["config"]["workload"] == "fluid4k" and d["config"]["particles"] == 4000
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_committed_traffic_follows_the_list_form():
    """The roofline's traffic comes from the committed ncu summary of the
    kernel that the list form runs, and the workload config names an explicit
    list form (the same dict on both arms)."""
    sys.path.insert(0, ROOT)
    import argparse

    import bench

    per_particle = bench.ncu_traffic("melt2m", False)
    slices = bench.ncu_traffic("melt2m", True)
    assert per_particle and slices and slices < 0.5 * per_particle
    base = dict(workload="melt2m", vs_com="fixed")
    assert "verlet_lists" not in bench.workload_config(argparse.Namespace(list_form="auto", **base), 2000000)
    cfg = bench.workload_config(argparse.Namespace(list_form="slice", **base), 2000000)
    assert "slice" in cfg["verlet_lists"]
