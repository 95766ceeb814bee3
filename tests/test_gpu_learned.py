"""The learned preconditioner on the GPU, through the C ABI.

* The hand-written forward and backward kernels against the CPU oracle
  (oracle/mpnn_ref.py) on a Newton system the simulator produced, with the
  same weights and probe vectors: loss within 1e-4 relative, gradient within
  1e-3 relative in norm (FP32 accumulation in different orders; the weights
  are BF16 on both sides, and so are the inputs of the message-passing
  layers, which run on the tensor cores).
* Training on systems the simulator produces lowers the loss, and the trained
  network cuts PCG iterations against block-Jacobi at the same 1e-6 residual
  while the trajectory stays within 1e-6 of the bounding-box diagonal.
"""
import numpy as np
import pytest

import cipc
import mpnn_ref as M

pytestmark = pytest.mark.gpu

LOSS_RTOL = 1e-4
GRAD_RTOL = 1e-3


def _oracle_system(d, btype):
    return M.System(d["nv"], d["rowPtr"], d["col"], d["val"], d["dRowS"], d["dRowE"], d["dCol"], d["dVal"], d["diagExtra"], btype)


def _weights(seed=3):
    w = M.init_weights(1).astype(np.float64)
    rng = np.random.default_rng(seed)
    w[M.WD:M.BD] = 0.05 * rng.standard_normal(M.BD - M.WD)
    w[M.WO:M.BO] += 0.05 * rng.standard_normal(M.BO - M.WO)
    w[M.BO:M.NPARAM] = 0.01 * rng.standard_normal(9)
    return w.astype(np.float32)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_loss_and_gradient_match_oracle(precision):
    sc = cipc.scene_two_cubes(3, gap=0.002)
    sim = cipc.Simulator(sc, precision=precision, precond="learned")
    for _ in range(4):
        sim.step()
    sim.assemble()
    d = sim.export_bsr()
    assert len(d["dCol"]) > 0, "the system should carry contact blocks"
    s = _oracle_system(d, sc["btype"])
    w = _weights()
    sim.set_precond_weights(w)
    probes = M.probe_vectors(s.nv, 3, 5).astype(np.float32)
    loss_g, grad_g = sim.precond_loss(probes=probes, grad=True)
    loss_o, grad_o = M.loss_and_grad(s, w, probes.astype(np.float64))
    assert abs(loss_g - loss_o) <= LOSS_RTOL * abs(loss_o), (loss_g, loss_o)
    err = np.linalg.norm(grad_g - grad_o) / np.linalg.norm(grad_o)
    assert err <= GRAD_RTOL, err
    # every parameter group is exercised and agrees
    for a, b in [(M.WN0, M.WE0), (M.WE0, M.LAYERS), (M.We(0), M.Wh(0)), (M.Wh(2), M.WD), (M.WD, M.WO), (M.WO, M.NPARAM)]:
        n = np.linalg.norm(grad_o[a:b])
        assert n > 0
        assert np.linalg.norm(grad_g[a:b] - grad_o[a:b]) <= 1e-2 * n
    # the device probe generator is the oracle's
    l_dev, _ = sim.precond_loss(nprobes=3, seed=5)
    assert abs(l_dev - loss_o) <= LOSS_RTOL * abs(loss_o)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_trained_network_beats_block_jacobi(precision):
    sc = cipc.scene_cloth_drape(32, 4, newton_thr=1e-6)
    jac = cipc.Simulator(sc, precision=precision, precond="jacobi")
    lrn = cipc.Simulator(sc, precision=precision, precond="learned")
    first = last = None
    # train on the Newton systems of the first steps (online, one system per step)
    for k in range(8):
        jac.step()
        lrn.step()
        a, b = lrn.precond_train(60, probes=4, lr=2e-3, seed=100 + k)
        first = a if first is None else first
        last = b
    assert last < first
    it_j = it_l = 0
    for k in range(6):
        it_j += jac.step()["pcgIterations"]
        it_l += lrn.step()["pcgIterations"]
    assert it_l < 0.8 * it_j, (it_l, it_j)
    assert lrn.precond_stats()["fallbacks"] == 0
    bbox = np.linalg.norm(np.asarray(sc["bbox_max"]) - np.asarray(sc["bbox_min"]))
    assert np.abs(lrn.get("x") - jac.get("x")).max() <= 1e-6 * bbox


def _to_slots(d, s, Gd, Ge):
    """Oracle factor (per vertex / per lower edge) in the device's slot layout."""
    nv = d["nv"]
    rp, col = d["rowPtr"], d["col"]
    ns, nd = len(col), len(d["dCol"])
    gs = np.zeros((ns, 3, 3)); gd = np.zeros((max(nd, 1), 3, 3))
    spos = {}
    for i in range(nv):
        for k in range(rp[i], rp[i + 1]):
            spos[(i, int(col[k]))] = k
    dpos = {}
    for i in range(nv):
        for k in range(d["dRowS"][i], d["dRowE"][i]):
            dpos[(i, int(d["dCol"][k]))] = k
    for i in range(nv):
        gs[spos[(i, i)]] = Gd[i]
    for e in range(s.E):
        i, j = int(s.ei[e]), int(s.ej[e])
        if s.edge_contact[e]:
            gd[dpos[(i, j)]] = Ge[e]
            if (j, i) in dpos:
                gd[dpos[(j, i)]] = Ge[e].T
        else:
            gs[spos[(i, j)]] = Ge[e]
            gs[spos[(j, i)]] = Ge[e].T
    return gs.reshape(-1, 9), gd[:nd].reshape(-1, 9)


@pytest.mark.parametrize("scene_name", ["two_cubes", "cloth_on_fixed_cube"])
def test_factors_match_oracle(scene_name):
    if scene_name == "two_cubes":
        sc = cipc.scene_two_cubes(3, gap=0.002)
        nsteps = 4
    else:
        sc = cipc.scene_cloth_drape(24, 3, newton_thr=1e-6)
        sc["x"] = sc["x"].copy()
        nsteps = 2
    sim = cipc.Simulator(sc, precision="mixed", precond="fsai")
    for _ in range(nsteps):
        sim.step()
    sim.assemble()
    d = sim.export_bsr()
    s = _oracle_system(d, sc["btype"])
    # the exact FSAI
    gs, gd = sim.precond_factor("fsai")
    es, ed = _to_slots(d, s, *M.fsai(s))
    scale = np.abs(es).max()
    assert np.abs(gs - es).max() <= 1e-5 * scale
    if len(ed):
        assert np.abs(gd - ed).max() <= 1e-5 * scale
    # the network forward (trained-looking weights).  The message-passing
    # layers round their inputs to BF16 on both sides, but the GPU forms
    # those inputs in FP32 and the oracle in FP64, so an input that lies
    # within rounding distance of a BF16 tie can round to the neighbouring
    # BF16 value: that input moves by 2^-8 of itself, and the entries
    # downstream of it by up to about 1e-3 of the factor's scale.  The bulk
    # of the entries agrees to FP32 accumulation order.
    w = _weights()
    sim.set_precond_weights(w)
    gs, gd = sim.precond_factor("learned")
    Gd, Ge, _ = M.forward(s, w)
    es, ed = _to_slots(d, s, Gd, Ge)
    scale = np.abs(es).max()
    diff = np.abs(np.concatenate([(gs - es).ravel(), (gd - ed).ravel()]))
    assert diff.max() <= 2e-3 * scale, (diff.max() / scale, np.median(diff) / scale)
    assert np.median(diff) <= 1e-6 * scale, (diff.max() / scale, np.median(diff) / scale)
    assert np.mean(diff <= 1e-4 * scale) >= 0.95, np.mean(diff <= 1e-4 * scale)


def test_fsai_pcg_cuts_iterations():
    sc = cipc.scene_cloth_drape(32, 4, newton_thr=1e-6)
    jac = cipc.Simulator(sc, precision="mixed", precond="jacobi")
    fs = cipc.Simulator(sc, precision="mixed", precond="fsai")
    it_j = it_f = 0
    for _ in range(10):
        it_j += jac.step()["pcgIterations"]
        it_f += fs.step()["pcgIterations"]
    assert it_f < 0.5 * it_j, (it_f, it_j)
    bbox = np.linalg.norm(np.asarray(sc["bbox_max"]) - np.asarray(sc["bbox_min"]))
    assert np.abs(fs.get("x") - jac.get("x")).max() <= 1e-6 * bbox
