"""bench.py --impl reference on the host cores, no GPU: one JSON line with the
metric, unit and direction of the GPU arm, a cpu_baseline describing the run
and an e2e entry without host-device copies.  A small cloth without settle
steps keeps it short (it starts from frame 0 and steps to the first timed
frame: saved contact states exist for the bench sizes only); the restore of
a saved state is covered by test_oracle_state.py."""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BENCH = os.path.join(HERE, "..", "bench.py")


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, BENCH, "--impl", "reference", "--scene", "cloth_drape", "--cloth", "16", "--settle-steps", "0",
                        "--steps", "2", "--warmup", "3"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "steps/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["config"]["workload"].startswith("cloth_drape_16")
    assert d["config"]["timed_frames"] == "3-4"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "from the start of the scene" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
