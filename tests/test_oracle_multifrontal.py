"""The oracle's multifrontal Cholesky (the PARDISO-class direct solver of
bench.py's CPU legs) against dense solves, across thread counts, and against
the oracle's envelope Cholesky on a cloth contact system."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "cpu-ipc_b200"))

import cipc  # noqa: E402
import oracle  # noqa: E402


def _lower_csr(A):
    n = A.shape[0]
    rp, col, val = [0], [], []
    for r in range(n):
        for c in range(r + 1):
            if A[r, c] != 0.0:
                col.append(c)
                val.append(A[r, c])
        rp.append(len(col))
    return np.array(rp, np.int32), np.array(col, np.int32), np.array(val)


def _spd_on_graph(nv, edges, rng):
    """SPD 3nv x 3nv matrix with a 3x3 block per graph edge."""
    A = np.zeros((3 * nv, 3 * nv))
    for (i, j) in edges:
        B = rng.standard_normal((3, 3))
        A[3 * i:3 * i + 3, 3 * j:3 * j + 3] += B
        A[3 * j:3 * j + 3, 3 * i:3 * i + 3] += B.T
    # diagonally dominant by blocks
    for i in range(nv):
        A[3 * i:3 * i + 3, 3 * i:3 * i + 3] += (np.abs(A[3 * i:3 * i + 3]).sum() + 1.0) * np.eye(3)
    return A


def _grid_two_ring(k):
    idx = lambda a, b: a * k + b  # noqa: E731
    e = set()
    for a in range(k):
        for b in range(k):
            for da, db in ((0, 1), (1, 0), (1, 1), (0, 2), (2, 0), (1, -1)):
                a2, b2 = a + da, b + db
                if 0 <= a2 < k and 0 <= b2 < k:
                    e.add((idx(a, b), idx(a2, b2)))
    return k * k, sorted(e)


def _graphs():
    rng = np.random.default_rng(7)
    yield "grid", _grid_two_ring(14)
    n = 180
    yield "random", (n, sorted({tuple(sorted(rng.choice(n, 2, replace=False))) for _ in range(500)}))
    # components of many sizes and isolated vertices (fixed vertices of a scene)
    parts, off, e = [1, 1, 2, 5, 30, 60, 3, 1], 0, []
    for s in parts:
        e += [(off + i, off + i + 1) for i in range(s - 1)]
        off += s
    yield "components", (off, e)
    yield "clique", (40, [(i, j) for i in range(40) for j in range(i + 1, 40)])
    yield "single", (1, [])


@pytest.mark.parametrize("name,graph", list(_graphs()))
def test_multifrontal_matches_dense_solve(name, graph):
    nv, edges = graph
    rng = np.random.default_rng(len(edges) + nv)
    A = _spd_on_graph(nv, edges, rng)
    b = rng.standard_normal(3 * nv)
    rp, col, val = _lower_csr(A)
    x_ref = np.linalg.solve(A, b)
    # orderings without positions (level sets) and with them (coordinate cuts)
    for xyz in (None, rng.random((nv, 3))):
        sols = []
        for threads in (1, 3, 8):
            x, _, _ = oracle.linear_solve(nv, rp, col, val, b, method="multifrontal", threads=threads, xyz=xyz)
            assert np.abs(x - x_ref).max() <= 1e-10 * np.abs(x_ref).max(), (name, threads)
            sols.append(x)
        # every entry takes its updates in pivot order whatever the thread count
        assert all(np.array_equal(sols[0], s) for s in sols[1:])


def test_multifrontal_rejects_an_indefinite_matrix():
    nv, edges = _grid_two_ring(6)
    A = _spd_on_graph(nv, edges, np.random.default_rng(1))
    A[40, 40] = -A[40, 40]
    rp, col, val = _lower_csr(A)
    with pytest.raises(RuntimeError):
        oracle.linear_solve(nv, rp, col, val, np.ones(3 * nv), method="multifrontal", threads=4)


def test_multifrontal_agrees_with_envelope_cholesky_on_a_contact_system():
    # a 24x24 cloth over the cube: in contact from about step 29
    o = oracle.Oracle(cipc.scene_cloth_drape(24, 4), linear="multifrontal", threads=4)
    for _ in range(34):
        st = o.step()
    assert st["selfContacts"] > 0
    o.friction_init()
    _, rp, col, val, rhs = o.system()
    x_mf, _, _ = oracle.linear_solve(o.nv, rp, col, val, rhs, method="multifrontal", threads=8)
    x_env, _, _ = oracle.linear_solve(o.nv, rp, col, val, rhs, method="direct")
    assert np.abs(x_mf - x_env).max() <= 1e-9 * np.abs(x_env).max()
