"""The learned preconditioner's CPU oracle (oracle/mpnn_ref.py), checked on
its own: analytic backward against central finite differences, BF16
rounding against torch's, and the two factor identities the design rests on
(G = I reproduces block-Jacobi; the initial weights give the first-order
factor G = I - strict_lower(Â)).  No GPU needed."""
import numpy as np
import pytest
import scipy.sparse as sp

import mpnn_ref as M


def _system(oracle_mod, cipc_mod, steps=3):
    """A small Newton system produced by the FP64 oracle (two stacked cubes in
    contact), as the static-only block layout the network reads."""
    sc = cipc_mod.scene_two_cubes(2, gap=0.002)
    o = oracle_mod.Oracle(sc, linear="direct")
    for _ in range(steps):
        o.step()
    _, rp, col, val, rhs = o.system()
    nv = o.nv
    n = 3 * nv
    L = sp.csr_matrix((val, col, rp), shape=(n, n))
    A = (L + L.T - sp.diags(L.diagonal())).tobsr(blocksize=(3, 3))
    A.sort_indices()
    z = np.zeros(nv, np.int64)
    s = M.System(nv, A.indptr, A.indices, A.data.reshape(-1, 9), z, z, np.zeros(0, np.int64), np.zeros((0, 9)), np.zeros((nv, 9)))
    return s, rhs.reshape(nv, 3)


def _weights(seed=3):
    w = M.init_weights(1).astype(np.float64)
    rng = np.random.default_rng(seed)
    # move the heads off their initial values so every layer gets a gradient
    w[M.WD:M.BD] = 0.05 * rng.standard_normal(M.BD - M.WD)
    w[M.WO:M.BO] += 0.05 * rng.standard_normal(M.BO - M.WO)
    w[M.BO:M.NPARAM] = 0.01 * rng.standard_normal(9)
    return w


@pytest.mark.parametrize("kind", ["kaporin", "residual"])
def test_backward_matches_finite_differences(oracle_mod, cipc_mod, monkeypatch, kind):
    s, _ = _system(oracle_mod, cipc_mod)
    monkeypatch.setattr(M, "bf16", lambda x: np.asarray(x, np.float64))  # exact weights for the FD check
    w = _weights()
    probes = M.probe_vectors(s.nv, 2, 11)
    _, g = M.loss_and_grad(s, w, probes, kind=kind)
    rng = np.random.default_rng(0)
    blocks = [(M.WN0, M.BN0), (M.WE0, M.BE0), (M.We(0), M.Be(0)), (M.Wh(1), M.Bh(1)), (M.We(2), M.Be(2)), (M.WD, M.BD), (M.WO, M.BO),
              (M.BD, M.WO), (M.Bh(2), M.Bh(2) + M.H)]
    checked = 0
    for a, b in blocks:
        for i in rng.choice(np.arange(a, b), 3, replace=False):
            h = 1e-6
            wp = w.copy(); wp[i] += h
            wm = w.copy(); wm[i] -= h
            fd = (M.loss_and_grad(s, wp, probes, False, kind)[0] - M.loss_and_grad(s, wm, probes, False, kind)[0]) / (2 * h)
            assert abs(fd - g[i]) <= 1e-5 * max(1e-3, abs(fd)) + 1e-9, (i, fd, g[i])
            checked += abs(g[i]) > 0
    assert checked >= 10  # the check saw non-trivial gradients in most layers


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    x = np.random.default_rng(0).standard_normal(10000).astype(np.float32) * np.float32(3.0)
    x[:4] = [1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -(1.0 + 2 ** -8), 0.0]  # ties to even
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(M.bf16(x), ref)


def test_identity_factor_is_block_jacobi(oracle_mod, cipc_mod):
    s, _ = _system(oracle_mod, cipc_mod)
    Gd = np.tile(np.eye(3), (s.nv, 1, 1))
    Ge = np.zeros((s.E, 3, 3))
    r = np.random.default_rng(1).standard_normal((s.nv, 3))
    z = M.precond_apply(s, Gd, Ge, r)
    assert np.allclose(z, M.block_jacobi(s)(r), rtol=1e-10, atol=1e-14 * np.abs(z).max())
    # the scaled matrix has identity diagonal blocks
    d = np.einsum("iab,ibc,idc->iad", s.S, s.D, s.S)
    assert np.allclose(d, np.eye(3), atol=1e-10)


def test_initial_weights_give_first_order_factor(oracle_mod, cipc_mod):
    s, b = _system(oracle_mod, cipc_mod)
    Gd, Ge, _ = M.forward(s, M.init_weights(1))
    assert np.allclose(Ge.reshape(-1, 9), -s.g, rtol=1e-6, atol=1e-7)
    assert np.allclose(Gd, np.eye(3), atol=4e-3)  # softplus(bf16(softplus^-1(1)))
    # it is already a better preconditioner than block-Jacobi on this system
    it_bj = M.pcg_iterations(s, b, M.block_jacobi(s))
    it_g = M.pcg_iterations(s, b, lambda r: M.precond_apply(s, Gd, Ge, r))
    assert it_g <= it_bj
