"""The hook at the linear-solve seam (NewtonLinearSystem::solve): every
Newton system written to disk matches the system the library holds, and
online training takes its Adam steps on every system as it arises."""
import glob
import os

import numpy as np
import pytest

import cipc

pytestmark = pytest.mark.gpu


def _in_contact(sim, steps=40):
    for _ in range(steps):
        st = sim.step()
        if st["selfContacts"] > 0:
            return st
    raise AssertionError("no contact")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dumped_system_matches_the_library(tmp_path, precision):
    sc = cipc.scene_cloth_drape(10, 2)
    sim = cipc.Simulator(sc, precision=precision)
    _in_contact(sim)
    sim.set_system_dump(tmp_path)
    st = sim.step()
    sim.set_system_dump(None)
    files = sorted(glob.glob(os.path.join(tmp_path, "system_*.bin")))
    # every assembled system: each barrier sub-problem's Newton steps and its confirming assembly
    assert len(files) == st["newtonIterations"] + st["kappaIterations"]
    last = cipc.read_system(files[-1])
    ex = sim.export_bsr()
    assert np.array_equal(last["row_ptr"], ex["rowPtr"]) and np.array_equal(last["col"], ex["col"])
    assert np.array_equal(last["val"].reshape(-1).astype(np.float64), ex["val"].reshape(-1))
    assert np.array_equal(last["diag_extra"].reshape(-1), ex["diagExtra"].reshape(-1))
    assert np.array_equal(last["dyn_row_start"], ex["dRowS"]) and np.array_equal(last["dyn_row_end"], ex["dRowE"])
    nd = len(last["dyn_col"])
    assert nd == len(ex["dCol"]) and nd > 0
    assert np.array_equal(last["dyn_col"], ex["dCol"])
    assert np.array_equal(last["dyn_val"].reshape(-1).astype(np.float64), ex["dVal"].reshape(-1))
    assert np.array_equal(last["btype"], sc["btype"])
    assert np.isfinite(last["rhs"]).all() and np.abs(last["rhs"]).max() > 0
    sim.close()


def test_online_training_sees_every_system():
    sc = cipc.scene_cloth_drape(10, 2)
    sim = cipc.Simulator(sc, precision="mixed", precond="learned")
    _in_contact(sim)
    w0 = sim.precond_weights()
    sim.set_online_training(3, probes=4, lr=1e-3, seed=5)
    newton = 0
    for _ in range(2):
        st = sim.step()
        newton += st["newtonIterations"] + st["kappaIterations"]
    assert sim.hook_systems() == newton
    assert sim.precond_stats()["adam_steps"] >= 3 * newton
    assert not np.array_equal(w0, sim.precond_weights())
    sim.close()
