"""Saved oracle states: bench.py's CPU legs restore one to time contact frames.

A restored state must continue exactly as the uninterrupted run does, must
refuse a scene it was not saved from, and the committed cloth-drape state must
still belong to the scene generator's cloth drape.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "cpu-ipc_b200"))

import cipc  # noqa: E402
import oracle  # noqa: E402


def test_restore_continues_bit_exactly(tmp_path):
    # a 16x16 cloth falls 0.1 m onto the cube: contact from about step 28
    scene = cipc.scene_cloth_drape(16, 10)
    ref = oracle.Oracle(scene, linear="pcg", threads=1)
    for _ in range(30):
        ref.step()
    path = str(tmp_path / "s.npz")
    ref.save_state(path, 30)
    kappa = ref.scalars()["kappa"]
    stats_ref = [ref.step() for _ in range(4)]
    assert stats_ref[-1]["groundContacts"] + stats_ref[-1]["selfContacts"] > 0

    o = oracle.Oracle(scene, linear="pcg", threads=1)
    assert o.restore_state(path) == 30
    assert o.scalars()["kappa"] == kappa
    stats = [o.step() for _ in range(4)]
    assert np.array_equal(o.get("x"), ref.get("x"))
    assert np.array_equal(o.get("vel"), ref.get("vel"))
    assert [s["newton"] for s in stats] == [s["newton"] for s in stats_ref]
    assert [s["pcgIterations"] for s in stats] == [s["pcgIterations"] for s in stats_ref]


def test_restore_refuses_another_scene(tmp_path):
    a = oracle.Oracle(cipc.scene_cloth_drape(16, 10), linear="pcg", threads=1)
    a.step()
    path = str(tmp_path / "s.npz")
    a.save_state(path, 1)
    b = oracle.Oracle(cipc.scene_cloth_drape(12, 10), linear="pcg", threads=1)
    with pytest.raises(ValueError):
        b.restore_state(path)


def test_save_needs_a_completed_step(tmp_path):
    a = oracle.Oracle(cipc.scene_cloth_drape(8, 4), linear="pcg", threads=1)
    a.step()
    a.set("vprev", a.get("x") + 1e-3)
    with pytest.raises(RuntimeError):
        a.save_state(str(tmp_path / "s.npz"), 1)


def test_committed_contact_state_matches_the_bench_scene():
    path = os.path.join(ROOT, "oracle", "states", "cloth_drape_128_frame40.npz")
    s = np.load(path)
    scene = cipc.scene_cloth_drape(128, 10)
    o = oracle.Oracle(scene, linear="pcg", threads=1)
    assert str(s["rest_sha256"]) == o.rest_digest()
    assert o.restore_state(path) == 40
    x = o.get("x")
    # the cube (the vertices after the cloth's) is fixed; the cloth is in
    # contact with it, below its starting height of 0.35 m
    cloth = np.arange(128 * 128)
    assert x[cloth, 1].min() < 0.35 - 0.05
    assert np.array_equal(x[128 * 128:], np.asarray(scene["x"]).reshape(-1, 3)[128 * 128:])
    assert np.isfinite(x).all() and np.isfinite(o.get("vel")).all()
