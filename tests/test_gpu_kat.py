"""The CUDA path on the reference's own demo scenes, against the answers the
reference's documentation quotes for them (tests/golden/kat_values.json):
twisting-mat (1 and 5 steps), twisting-mat-soft (5 steps) and cloth-bunny
(1 step), FP64, PCG at 1e-10 relative so that the linear solves are as exact
as the reference's direct solver.

The meshes are the reference's own, copied under tests/golden/assets.  Every
scene runs under both segment-triangle intersection rules (the reference's
exact rule and the default near-coplanar tolerance): the known answers hold
under either."""
import json
import os

import numpy as np
import pytest

import cipc
import ref_scenes

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_scenes.assets_available("twisting_mat") or not ref_scenes.assets_available("cloth_bunny"),
                                                  reason="reference assets not available")]
RULES = pytest.mark.parametrize("rule", ["tolerant", "reference"])

KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "kat_values.json")))


def _run(scene, steps, rule):
    sim = cipc.Simulator(scene, precision="fp64", precond="jacobi", tol=1e-10)
    sim.set_intersection_rule(rule)
    for _ in range(steps):
        st = sim.step()
    return sim.get("x"), st


@RULES
def test_twisting_mat_one_step(rule):
    x, st = _run(ref_scenes.twisting_mat(False), 1, rule)
    k = KAT["twisting_mat_1_step"]
    assert st["newtonIterations"] == k["newton"]
    assert abs((x ** 2).sum() - k["squared_norm_sum"]) <= 1e-12 * k["squared_norm_sum"]


@RULES
def test_twisting_mat_five_steps(rule):
    x, st = _run(ref_scenes.twisting_mat(False), 5, rule)
    k = KAT["twisting_mat_5_steps"]
    assert st["newtonIterations"] == k["newton_last"]
    ref = float(k["squared_norm_sum_prefix"])  # quoted to 12 decimals
    assert abs((x ** 2).sum() - ref) <= 1e-12 * ref


@RULES
def test_twisting_mat_soft_five_steps(rule):
    x, st = _run(ref_scenes.twisting_mat(True), 5, rule)
    k = KAT["twisting_mat_soft_5_steps"]
    assert st["newtonIterations"] == k["newton_last"]
    assert abs((x ** 2).sum() - k["squared_norm_sum"]) <= 1e-9 * k["squared_norm_sum"]


@RULES
def test_cloth_bunny_one_step(rule):
    _, st = _run(ref_scenes.cloth_bunny(), 1, rule)
    k = KAT["cloth_bunny_1_step"]
    assert st["newtonIterations"] == k["newton"]
    assert st["energyBacktracks"] == k["energy_backtracks"]
    assert st["intersectionBacktracks"] == k["intersection_backtracks"]
    assert abs(st["minConstraintDistance2"] - k["min_distance2"]) <= 1e-9 * k["min_distance2"]


@RULES
def test_cloth_bunny_hinge_bending_one_step(rule):
    _, st = _run(ref_scenes.cloth_bunny(hinge=True), 1, rule)
    k = KAT["cloth_bunny_hinge_1_step"]
    assert st["newtonIterations"] == k["newton"]
    assert st["energyBacktracks"] == k["energy_backtracks"]
    assert st["intersectionBacktracks"] == k["intersection_backtracks"]


@pytest.mark.skipif(not ref_scenes.assets_available("bunny2"), reason="bunny2 mesh not available")
def test_bunny2_one_step():
    """The two-bunny PARDISO benchmark scene (38,386 vertices, 159,870 tets):
    surface size and the documented Newton count of its first step."""
    sc = ref_scenes.bunny2()
    k = KAT["bunny2_1_step"]
    sim = cipc.Simulator(sc, precision="fp64", precond="jacobi", tol=1e-10)
    assert sim.counts()[1] == k["surface_faces"]
    st = sim.step()
    assert st["newtonIterations"] == k["newton"]
