"""The preconditioner network trained by the held-out protocol
(cpu-ipc_b200/train_precond.py: Newton systems of pile seeds 0-49) on a pile
it never saw (seed 55), in the contact phase: fewer PCG iterations per
Newton iteration than block-Jacobi, and its count beside the exact FSAI
factor of the same pattern (the optimum of its loss) recorded."""
import os

import numpy as np
import pytest

import cipc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WEIGHTS = os.path.join(ROOT, "cpu-ipc_b200", "weights", "pile_64x12_seeds0-49.bin")


def _restore(sim, state):
    for k in ("x", "vel", "vprev", "xtilde"):
        sim.set(k, state[k])
    sim.set_kappa(state["kappa"])
    sim.collision_sets()


def test_trained_network_beats_block_jacobi_on_an_unseen_pile():
    w = np.fromfile(WEIGHTS, np.float32)
    assert len(w) == cipc.lib().cipc_gpu_precond_num_params()
    sc = cipc.scene_pile(64, 12, seed=55)
    base = cipc.Simulator(sc, precision="fp64", precond="jacobi")
    for _ in range(30):
        base.step()
    state = {k: base.get(k) for k in ("x", "vel", "vprev", "xtilde")}
    state["kappa"] = base.scalars()["kappa"]
    base.close()
    per_newton = {}
    for pre in ("jacobi", "learned", "fsai"):
        sim = cipc.Simulator(sc, precision="mixed", precond=pre)
        if pre == "learned":
            sim.set_precond_weights(w)
        _restore(sim, state)
        newton = pcg = 0
        for _ in range(2):
            st = sim.step()
            newton += st["newtonIterations"]
            pcg += st["pcgIterations"]
        per_newton[pre] = pcg / max(1, newton)
        if pre != "jacobi":
            assert sim.precond_stats()["fallbacks"] == 0
        sim.close()
    print("PCG iterations per Newton iteration, seed 55:", per_newton)
    assert per_newton["learned"] < per_newton["jacobi"]
