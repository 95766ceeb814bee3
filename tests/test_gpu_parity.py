"""Parity of the CUDA path (through the C ABI) against the FP64 oracle.

Bars, as the task sets them: contact pair sets bit-exact; energy, gradient
and Hessian within 1e-10 relative in FP64; CCD time of impact within 1e-6
relative and never above the oracle's conservative step; trajectories within
1e-6 of the bounding-box diagonal after N steps at the same Newton tolerance.
Mixed precision (FP32 element/friction blocks and SpMV) is held to the FP32
round-off of those blocks and to the same trajectory bar.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import cipc

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-10
HESS_TOL = 1e-10
ENERGY_TOL = 1e-10
TRAJ_TOL = 1e-6


def _pair(oracle_mod, scene, linear="direct", **kw):
    o = oracle_mod.Oracle(scene, linear=linear)
    g = cipc.Simulator(scene, surface=o.surface(), **kw)
    return o, g


def _perturb(o, g, scene, scale, seed=0, vel=0.0):
    rng = np.random.default_rng(seed)
    free = (scene["btype"] == 0)[:, None]
    x = o.get("x") + scale * rng.standard_normal((o.nv, 3)) * free
    o.set("x", x)
    g.set("x", x)
    if vel:
        v = vel * rng.standard_normal((o.nv, 3)) * free
        o.set("vel", v); g.set("vel", v)
        vp = o.get("vprev")
        xt = vp + v * scene["params"]["dt"] + np.array([0, -9.8 * scene["params"]["dt"] ** 2, 0]) * scene["params"].get("apply_gravity", 1)
        o.set("xtilde", xt); g.set("xtilde", xt)
    return x


def _canon(S):
    return [sorted(map(tuple, S[k].tolist())) for k in ("self_active", "self_ee", "ccd")] + [sorted(S["ground"].tolist())]


def _oracle_full_matrix(rp, col, val, n):
    L = sp.csr_matrix((val, col, rp), shape=(n, n))
    return (L + L.T - sp.diags(L.diagonal())).tocsr()


def _gpu_full_matrix(g, btype):
    r, c, v = g.export_matrix()
    n = 3 * g.nv
    A = sp.coo_matrix((v, (r, c)), shape=(n, n)).tocsr()
    free = np.repeat(btype == 0, 3)
    D = sp.diags(free.astype(float))
    return (D @ A @ D + sp.diags((~free) * A.diagonal())).tocsr()


def _hinge(sc):
    """The scene with dihedral-angle hinge bending in place of quadratic bending."""
    sc["params"] = dict(sc["params"], quad_bending=2)
    return sc


CONTACT_SCENES = {
    "cubes_touching": lambda: (cipc.scene_two_cubes(3, gap=0.0015), 2e-4),
    "cloth_on_cube": lambda: (cipc.scene_cloth_drape(10, 2), 0.0),
    "cloth_on_cube_hinge": lambda: (_hinge(cipc.scene_cloth_drape(10, 2)), 0.0),
    "pile": lambda: (cipc.scene_pile(4, 2, seed=3), 0.0),
}


@pytest.fixture(scope="module")
def contact_states(oracle_mod):
    """States with many live contacts: run the oracle until contacts appear."""
    out = {}
    for name, make in CONTACT_SCENES.items():
        sc, pert = make()
        o = oracle_mod.Oracle(sc, linear="direct")
        if pert:
            rng = np.random.default_rng(7)
            o.set("x", o.get("x") + pert * rng.standard_normal((o.nv, 3)) * (sc["btype"] == 0)[:, None])
        else:
            for _ in range(60):
                st = o.step()
                if st["selfContacts"] + st["groundContacts"] > 8:
                    break
        out[name] = (sc, o.get("x"), o.get("vprev"), o.get("vel"), o.get("xtilde"), o.scalars()["kappa"] or 1e3)
    return out


@pytest.mark.parametrize("name", list(CONTACT_SCENES))
def test_active_sets_bit_exact(oracle_mod, contact_states, name):
    sc, x, vp, vel, xt, kappa = contact_states[name]
    o, g = _pair(oracle_mod, sc)
    for f, a in (("x", x), ("vprev", vp), ("vel", vel), ("xtilde", xt)):
        o.set(f, a); g.set(f, a)
    So, Sg = o.collision_sets(), g.collision_sets()
    co, cg = _canon(So), _canon(Sg)
    assert len(co[2]) > 0
    for a, b in zip(co, cg):
        assert a == b
    # ordering: same canonical order as the reference lists
    assert np.array_equal(So["self_active"], Sg["self_active"])
    assert np.array_equal(So["ccd"], Sg["ccd"])


@pytest.mark.parametrize("name", list(CONTACT_SCENES))
def test_gradient_hessian_energy(oracle_mod, contact_states, name):
    sc, x, vp, vel, xt, kappa = contact_states[name]
    o, g = _pair(oracle_mod, sc)
    for f, a in (("x", x), ("vprev", vp), ("vel", vel), ("xtilde", xt)):
        o.set(f, a); g.set(f, a)
    o.set_kappa(kappa); g.set_kappa(kappa)
    o.collision_sets(); g.collision_sets()
    o.friction_init(); g.friction_init()
    # move a little so friction has a non-zero tangential displacement
    x2 = _perturb(o, g, sc, 1e-5, seed=11)
    o.collision_sets(); g.collision_sets()
    go, rp, col, val, rhs = o.system()
    gg, _ = g.assemble()
    scale = np.abs(go).max()
    assert scale > 0
    assert np.abs(go - gg).max() <= GRAD_TOL * scale
    n = 3 * o.nv
    Ao = _oracle_full_matrix(rp, col, val, n)
    Ag = _gpu_full_matrix(g, sc["btype"])
    assert abs(Ao - Ag).max() <= HESS_TOL * abs(Ao).max()
    for k in (kappa, 2 * kappa):
        eo, eg = o.energy(k), g.energy(k)
        assert abs(eo - eg) <= ENERGY_TOL * abs(eo)


def test_elastic_gradient_hessian_away_from_rest(oracle_mod):
    sc = cipc.scene_twist(2, 8, 6)
    o, g = _pair(oracle_mod, sc)
    _perturb(o, g, sc, 5e-3, seed=5, vel=0.3)
    go, rp, col, val, rhs = o.system()
    gg, _ = g.assemble()
    assert np.abs(go - gg).max() <= GRAD_TOL * np.abs(go).max()
    Ao = _oracle_full_matrix(rp, col, val, 3 * o.nv)
    Ag = _gpu_full_matrix(g, sc["btype"])
    assert abs(Ao - Ag).max() <= HESS_TOL * abs(Ao).max()
    assert abs(o.energy(0.0) - g.energy(0.0)) <= ENERGY_TOL * abs(o.energy(0.0))


@pytest.mark.parametrize("name", list(CONTACT_SCENES))
def test_ccd_and_step_bounds(oracle_mod, contact_states, name):
    sc, x, vp, vel, xt, kappa = contact_states[name]
    o, g = _pair(oracle_mod, sc)
    for f, a in (("x", x), ("vprev", vp), ("vel", vel), ("xtilde", xt)):
        o.set(f, a); g.set(f, a)
    o.collision_sets(); g.collision_sets()
    rng = np.random.default_rng(2)
    d = rng.standard_normal((o.nv, 3)) * 0.05 * (sc["btype"] == 0)[:, None]
    d[:, 1] = np.abs(d[:, 1])  # push toward the ground and into contacts
    bo = o.step_bounds(d, 1.0)
    bg = g.step_bounds(d, 1.0)
    for k in ("ground", "partial", "cfl", "full"):
        assert abs(bo[k] - bg[k]) <= 1e-6 * abs(bo[k]), k
        assert bg[k] <= bo[k] * (1 + 1e-12) + 1e-300, k


@pytest.mark.parametrize("scene_fn,steps", [
    (lambda: cipc.scene_two_cubes(3), 25),
    (lambda: cipc.scene_cloth_drape(10, 2), 25),
    (lambda: _hinge(cipc.scene_cloth_drape(10, 2)), 25),
    (lambda: cipc.scene_pile(4, 2, seed=3), 15),
    (lambda: cipc.scene_twist(2, 8, 6), 6),
])
def test_trajectory_fp64(oracle_mod, scene_fn, steps):
    sc = scene_fn()
    o, g = _pair(oracle_mod, sc, linear="pcg")
    bb = np.sqrt(o.scalars()["bboxDiag2"])
    for s in range(steps):
        so, sg = o.step(), g.step()
        err = np.abs(o.get("x") - g.get("x")).max() / bb
        assert err <= TRAJ_TOL, (s, err)


def test_trajectory_mixed_precision(oracle_mod):
    sc = cipc.scene_cloth_drape(10, 2)
    o, g = _pair(oracle_mod, sc, linear="pcg", precision="mixed")
    bb = np.sqrt(o.scalars()["bboxDiag2"])
    for s in range(20):
        o.step(); g.step()
    assert np.abs(o.get("x") - g.get("x")).max() / bb <= TRAJ_TOL


def test_mixed_precision_blocks_are_fp32_rounded(oracle_mod, contact_states):
    sc, x, vp, vel, xt, kappa = contact_states["cubes_touching"]
    o, g = _pair(oracle_mod, sc, precision="mixed")
    for f, a in (("x", x), ("vprev", vp), ("vel", vel), ("xtilde", xt)):
        o.set(f, a); g.set(f, a)
    o.set_kappa(kappa); g.set_kappa(kappa)
    o.collision_sets(); g.collision_sets()
    o.friction_init(); g.friction_init()
    go, rp, col, val, rhs = o.system()
    gg, _ = g.assemble()
    assert np.abs(go - gg).max() <= GRAD_TOL * np.abs(go).max()  # gradient stays FP64
    Ao = _oracle_full_matrix(rp, col, val, 3 * o.nv)
    Ag = _gpu_full_matrix(g, sc["btype"])
    assert abs(Ao - Ag).max() <= 1e-5 * abs(Ao).max()


def test_standalone_pcg_matches_direct_solve():
    rng = np.random.default_rng(0)
    nv = 200
    # random SPD block matrix on a ring graph
    blocks = {}
    for i in range(nv):
        for j in (i, (i + 1) % nv, (i + 7) % nv):
            B = rng.standard_normal((3, 3)) * 0.1
            blocks.setdefault((i, j), np.zeros((3, 3)))
            blocks[(i, j)] += B
            blocks.setdefault((j, i), np.zeros((3, 3)))
            blocks[(j, i)] += B.T
    for i in range(nv):
        blocks[(i, i)] += 4.0 * np.eye(3)
    keys = sorted(blocks)
    rp = np.zeros(nv + 1, np.int32)
    for (i, j) in keys:
        rp[i + 1] += 1
    rp = np.cumsum(rp).astype(np.int32)
    ci = np.array([j for (i, j) in keys], np.int32)
    vals = np.stack([blocks[k] for k in keys])
    A = sp.bsr_matrix((vals, ci, rp), shape=(3 * nv, 3 * nv)).tocsr()
    b = rng.standard_normal(3 * nv)
    for prec in ("fp64", "mixed"):
        x, it, rr = cipc.pcg_bsr(rp, ci, vals, b, precision=prec, tol=1e-8)
        assert np.linalg.norm(A @ x - b) <= 1e-6 * np.linalg.norm(b)
        assert it > 0


def test_step_statistics_match(oracle_mod):
    sc = cipc.scene_two_cubes(2)
    o, g = _pair(oracle_mod, sc, linear="pcg")
    for s in range(14):
        so, sg = o.step(), g.step()
        assert so["newton"] == sg["newtonIterations"]
        assert so["energyBacktracks"] == sg["energyBacktracks"]
        assert so["groundContacts"] == sg["groundContacts"]
        assert so["selfContacts"] == sg["selfContacts"]
        assert abs(so["kappa"] - sg["kappa"]) <= 1e-10 * abs(so["kappa"])
