"""Unit checks of the oracle's building blocks (no GPU): exact distance
derivatives against finite differences, the PSD projection of the Stable
Neo-Hookean Hessian, additive CCD conservativeness, and the active set built
through the LBVH against a brute-force pair enumeration."""
import numpy as np
import pytest

import cipc


def _fd(kind, pts, h=1e-6):
    import oracle
    d0, g0, H0 = oracle.distance(kind, pts)
    n = len(g0)
    p = np.asarray(pts, float).reshape(-1)
    gfd = np.zeros(n)
    Hfd = np.zeros((n, n))
    for i in range(n):
        e = np.zeros(n); e[i] = h
        dp, gp, _ = oracle.distance(kind, p + e)
        dm, gm, _ = oracle.distance(kind, p - e)
        gfd[i] = (dp - dm) / (2 * h)
        Hfd[:, i] = (gp - gm) / (2 * h)
    return g0, H0, gfd, Hfd


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
def test_distance_derivatives_match_finite_differences(oracle_mod, kind):
    rng = np.random.default_rng(kind)
    npt = {0: 2, 1: 3}.get(kind, 4)
    for _ in range(5):
        pts = rng.standard_normal((npt, 3))
        g, H, gfd, Hfd = _fd(kind, pts)
        assert np.allclose(g, gfd, rtol=1e-6, atol=1e-7 * max(1, np.abs(g).max()))
        assert np.allclose(H, Hfd, rtol=1e-5, atol=1e-6 * max(1, np.abs(H).max()))
        assert np.allclose(H, H.T, atol=1e-12 * max(1, np.abs(H).max()))


def test_snh_hessian_is_psd_projection(oracle_mod):
    rng = np.random.default_rng(3)
    u, r = 5e4, 2e5
    for _ in range(20):
        F = np.eye(3) + 0.6 * rng.standard_normal((3, 3))
        P, H, psi = oracle_mod.snh(F, u, r)
        w = np.linalg.eigvalsh(H)
        assert w.min() > -1e-9 * max(1.0, w.max())
        # PK1 is the derivative of the energy density
        h = 1e-6
        Pfd = np.zeros((3, 3))
        for i in range(3):
            for j in range(3):
                E = np.zeros((3, 3)); E[i, j] = h
                Pfd[i, j] = (oracle_mod.snh(F + E, u, r)[2] - oracle_mod.snh(F - E, u, r)[2]) / (2 * h)
        assert np.allclose(P, Pfd, rtol=1e-5, atol=1e-4)


def test_accd_is_conservative(oracle_mod):
    # a point falling through a triangle: TOI must stop short of the plane
    p = np.array([[0.2, 1.0, 0.2], [0, 0, 0], [1, 0, 0], [0, 0, 1]], float)
    d = np.array([[0, -2.0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]], float)
    t = oracle_mod.pt_ccd(p, d, 0.2)
    assert 0.0 < t < 0.5
    # separating motion gives the full step
    assert oracle_mod.pt_ccd(p, -d, 0.2) == 1.0
    a = np.array([[-1, 1, 0], [1, 1, 0], [0, 0, -1], [0, 0, 1]], float)
    da = np.array([[0, -2, 0], [0, -2, 0], [0, 0, 0], [0, 0, 0]], float)
    te = oracle_mod.ee_ccd(a, da, 0.2)
    assert 0.0 < te < 0.5


def _brute_pairs(x, faces, verts, edges, btype, gap):
    lo_f = x[faces].min(1); hi_f = x[faces].max(1)
    pt = set()
    for si, v in enumerate(verts):
        p = x[v]
        ok = ~((lo_f - p > gap).any(1) | (p - hi_f > gap).any(1))
        for f in np.nonzero(ok)[0]:
            F = faces[f]
            if v in F:
                continue
            if btype[v] >= 2 and (btype[F] >= 2).all():
                continue
            pt.add((-si - 1, int(f)))
    lo_e = x[edges].min(1); hi_e = x[edges].max(1)
    ee = set()
    for i in range(len(edges)):
        ok = ~((lo_e - hi_e[i] > gap).any(1) | (lo_e[i] - hi_e > gap).any(1))
        for j in np.nonzero(ok)[0]:
            if j <= i or len(set(edges[i]) & set(edges[j])):
                continue
            if (btype[edges[i]] >= 2).all() and (btype[edges[j]] >= 2).all():
                continue
            ee.add((i, int(j)))
    return pt | ee


def test_lbvh_candidates_equal_brute_force(oracle_mod):
    sc = cipc.scene_two_cubes(2, gap=0.002)
    o = oracle_mod.Oracle(sc)
    rng = np.random.default_rng(0)
    x = o.get("x") + 1e-3 * rng.standard_normal((o.nv, 3))
    o.set("x", x)
    s = o.collision_sets()
    faces, verts, edges = o.surface()
    gap = np.sqrt(o.scalars()["Hhat"]) * 30
    got = set(map(tuple, s["ccd"].tolist()))
    # the oracle's gap is sqrt(Hhat); rebuild the brute force with the same gap
    want = _brute_pairs(x, faces, verts, edges, sc["btype"], np.sqrt(o.scalars()["Hhat"]))
    assert got == want


def test_pile_scene_places_every_cube_apart():
    """The pile generator terminates at the configuration's size (64 cubes of
    0.2 m in a 1.5 m box) and no two cubes' bounding spheres overlap, so the
    initial state is free of intersections whatever the rotations."""
    sc = cipc.scene_pile(64, 2)
    x = sc["x"][sc["btype"] != 2].reshape(64, -1, 3)
    centers = x.mean(axis=1)
    radius = np.linalg.norm(x - centers[:, None, :], axis=2).max()
    d = np.linalg.norm(centers[:, None, :] - centers[None, :, :], axis=2)
    d[np.arange(64), np.arange(64)] = np.inf
    assert d.min() > 2 * radius
    # inside the box walls and above the floor
    assert x[..., 1].min() > -1.0 + 0.02 and np.abs(x[..., 0]).max() < 0.8 and np.abs(x[..., 2]).max() < 0.8
    # seeded: the same seed gives the same scene
    assert np.array_equal(cipc.scene_pile(64, 2)["x"], sc["x"])


def _rand_hinge(rng):
    """A hinge (edge start, edge end, two opposite vertices) near the unit
    square split along its diagonal, and a bent copy of it."""
    rest = np.array([[0, 0, 0], [1, 1, 0], [1, 0, 0], [0, 1, 0]], float) + 0.05 * rng.standard_normal((4, 3))
    x = rest + 0.2 * rng.standard_normal((4, 3))
    return x, rest


def test_hinge_gradient_and_hessian_match_finite_differences(oracle_mod):
    """The oracle's hinge element (energy 0.5 k w remainder(theta - theta0)^2,
    HingeBending.cpp:76-106): its gradient matches central differences of its
    energy, and its Hessian matches the PSD projection (clamped eigenvalues,
    as makePD) of the central-difference Hessian of the energy."""
    rng = np.random.default_rng(5)
    k = 3.0
    for _ in range(6):
        x, rest = _rand_hinge(rng)
        e, g, H = oracle_mod.hinge(x, rest, k)
        h = 1e-6
        gf = np.zeros(12)
        Hf = np.zeros((12, 12))
        for i in range(12):
            d = np.zeros(12); d[i] = h
            ep, gp, _ = oracle_mod.hinge(x.reshape(12) + d, rest, k)
            em, gm, _ = oracle_mod.hinge(x.reshape(12) - d, rest, k)
            gf[i] = (ep - em) / (2 * h)
            Hf[:, i] = (gp - gm) / (2 * h)
        assert np.abs(g - gf).max() <= 1e-6 * max(1.0, np.abs(g).max())
        # the finite differences of the projected gradient see the unprojected
        # Hessian; project it the way makePD does and compare
        w, V = np.linalg.eigh(0.5 * (Hf + Hf.T))
        Hp = (V * np.maximum(w, 0.0)) @ V.T
        assert np.abs(H - Hp).max() <= 1e-5 * max(1.0, np.abs(Hp).max())
        assert np.allclose(H, H.T) and np.linalg.eigvalsh(H).min() >= -1e-9 * np.abs(H).max()


def test_hinge_energy_invariants(oracle_mod):
    """Zero at the rest shape, unchanged by a rigid motion of the bent shape,
    and the same whichever opposite vertex is listed first."""
    rng = np.random.default_rng(6)
    x, rest = _rand_hinge(rng)
    e0, g0, _ = oracle_mod.hinge(rest, rest, 2.0)
    assert abs(e0) < 1e-20 and np.abs(g0).max() < 1e-12
    e, _, _ = oracle_mod.hinge(x, rest, 2.0)
    q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    er, _, _ = oracle_mod.hinge(x @ q.T + np.array([0.3, -1.0, 2.0]), rest, 2.0)
    assert abs(er - e) <= 1e-12 * abs(e)
    es, _, _ = oracle_mod.hinge(x[[0, 1, 3, 2]], rest[[0, 1, 3, 2]], 2.0)
    assert abs(es - e) <= 1e-12 * abs(e)


def test_exact_solve_steps_a_pile_of_rotated_cubes(oracle_mod):
    """With an exact linear solve the first free-fall step is an exact
    translation, which keeps the faces of the rotated cubes coplanar up to
    rounding; the intersection test must not report the edges and triangles
    of one face as intersecting (or the line search gives up at frame 0)."""
    sc = cipc.scene_pile(8, 12)
    o = oracle_mod.Oracle(sc, linear="multifrontal", threads=8)
    assert not o.intersected()
    for _ in range(2):
        st = o.step()
    assert st["intersectionBacktracks"] == 0
