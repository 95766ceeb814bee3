"""The candidate-pair buffer of the full CCD and of the intersection test on a
B200: when a tree walk finds more candidate pairs than the buffer holds, the
buffer grows and the pass runs again, so the step bounds, the intersection
test and whole steps come out the same as with a buffer that is large from
the start.  The 8-cube pile's saved contact state runs in two processes, one
with a 16-pair first buffer (CIPC_CCD_PAIRS_INITIAL, read once per process)
and one with the default, and the results must agree bit for bit (the
minimum time of impact and the intersection flag do not depend on the order
of the pairs)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import json, os, sys
import numpy as np
sys.path.insert(0, os.path.join(sys.argv[1], "cpu-ipc_b200"))
import cipc
sc = cipc.scene_pile(8, 12)
g = cipc.Simulator(sc)
s = np.load(os.path.join(sys.argv[1], "oracle", "states", "pile_8x12_frame60.npz"))
dt = sc["params"]["dt"]
x, vel = s["x"], s["vel"]
g.set("x", x); g.set("vprev", x); g.set("vel", vel)
g.set("xtilde", x + vel * dt + np.array([0.0, float(s["gravity"]) * dt * dt, 0.0]))
g.set_kappa(float(s["kappa"]))
g.collision_sets()
rng = np.random.default_rng(3)
d = rng.standard_normal(x.shape) * 0.01 * (sc["btype"] == 0)[:, None]
bounds = {k: float(v) for k, v in g.step_bounds(d, 1.0).items()}
inter = g.intersected()
steps = [g.step()["newtonIterations"] for _ in range(2)]
print(json.dumps({"bounds": bounds, "intersected": inter, "newton": steps, "x": g.get("x").tobytes().hex()}))
g.close()
"""


def _run(initial):
    env = dict(os.environ)
    env.pop("CIPC_CCD_PAIRS_INITIAL", None)
    if initial:
        env["CIPC_CCD_PAIRS_INITIAL"] = str(initial)
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_small_pair_buffer_gives_the_same_results():
    small, default = _run(16), _run(None)
    assert small["bounds"] == default["bounds"]
    assert small["intersected"] == default["intersected"] is False
    assert small["newton"] == default["newton"]
    assert small["x"] == default["x"]
    assert all(np.isfinite(v) for v in default["bounds"].values())
