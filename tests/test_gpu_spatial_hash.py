"""The spatial-hash broad phase (the reference's SpatialHash backend, kept as
an A/B alternative to the LBVH): the same contact sets as the LBVH and the
oracle, bit for bit, the same step bounds, and identical trajectories."""
import numpy as np
import pytest

import cipc

pytestmark = pytest.mark.gpu


def _canon(S):
    return [sorted(map(tuple, S[k].tolist())) for k in ("self_active", "self_ee", "ccd")] + [sorted(S["ground"].tolist())]


@pytest.mark.parametrize("make,steps", [
    (lambda: cipc.scene_cloth_drape(10, 2), 60),
    (lambda: cipc.scene_pile(4, 2, seed=3), 45),
    (lambda: cipc.scene_two_cubes(3, gap=0.002), 10),
])
def test_same_trajectory_as_lbvh(oracle_mod, make, steps):
    sc = make()
    o = oracle_mod.Oracle(sc, linear="direct")
    a = cipc.Simulator(sc, surface=o.surface())
    b = cipc.Simulator(sc, surface=o.surface())
    b.set_broad_phase("spatial-hash")
    contacts = 0
    for _ in range(steps):
        sa, sb = a.step(), b.step()
        assert sa["newtonIterations"] == sb["newtonIterations"]
        contacts = max(contacts, sa["selfContacts"])
        assert np.array_equal(a.get("x"), b.get("x"))
    assert contacts > 0
    # contact sets against the LBVH and the oracle at the final state
    o.set("x", a.get("x"))
    Sa, Sb, So = a.collision_sets(), b.collision_sets(), o.collision_sets()
    for u, v, w in zip(_canon(Sa), _canon(Sb), _canon(So)):
        assert u == v == w
    rng = np.random.default_rng(1)
    d = rng.standard_normal((a.nv, 3)) * 0.05 * (sc["btype"] == 0)[:, None]
    ba, bb = a.step_bounds(d, 1.0), b.step_bounds(d, 1.0)
    for k in ("ground", "partial", "cfl", "full"):
        assert ba[k] == bb[k], k
    a.close(); b.close()
