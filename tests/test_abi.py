"""The C-ABI library builds, loads without a GPU, exports every entry point
include/cipc_gpu.h declares, and rejects bad input before touching a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import cipc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "cipc_gpu.h")).read()
    return sorted(set(re.findall(r"\b(cipc_gpu_\w+)\s*\(", src)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(cipc.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    L = C.CDLL(cipc.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(L, name), name


def _create(scene, opts):
    L = cipc.lib()
    d, keep = cipc.scene_desc(scene)
    h = C.c_void_p()
    rc = L.cipc_gpu_create(C.byref(d), C.byref(opts) if opts is not None else None, C.byref(h))
    return rc, h, L.cipc_gpu_create_error().decode()


def test_create_rejects_empty_scene():
    L = cipc.lib()
    d = cipc.SceneDesc()
    h = C.c_void_p()
    assert L.cipc_gpu_create(C.byref(d), None, C.byref(h)) == 1
    assert not h.value
    assert "vertices" in L.cipc_gpu_create_error().decode()


def test_create_rejects_out_of_range_index():
    sc = cipc.scene_two_cubes(1)
    sc["tets"] = sc["tets"].copy()
    sc["tets"][0, 0] = 10_000
    rc, h, msg = _create(sc, cipc.linear_options())
    assert rc == 1 and not h.value and "out-of-range" in msg


def test_create_rejects_cpu_backends():
    sc = cipc.scene_two_cubes(1)
    opts = cipc.LinearOptions(1, 0, 0, 1e-6, 100)  # LinearSolverBackend::Pardiso
    rc, h, msg = _create(sc, opts)
    assert rc == 1 and "GPU PCG" in msg


def test_create_rejects_free_dirichlet_vertex():
    sc = cipc.scene_twist(2, 8, 4)
    sc["btype"] = sc["btype"].copy()
    sc["btype"][sc["dirichlet"]["idx"][0]] = 0
    rc, h, msg = _create(sc, cipc.linear_options())
    assert rc == 1 and "Dirichlet" in msg


def test_no_cpu_fallback_without_device():
    """Without a CUDA device the library reports a CUDA error instead of
    silently computing on the host."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    rc, h, msg = _create(cipc.scene_two_cubes(1), cipc.linear_options())
    assert rc == 3 and not h.value


def test_create_rejects_unknown_bending_model():
    sc = cipc.scene_cloth_drape(4, 1)
    sc["params"] = dict(sc["params"], quad_bending=3)
    rc, h, msg = _create(sc, cipc.linear_options())
    assert rc == 1 and not h.value and "bending model" in msg


def _small_block_system(nv=6):
    cols = [sorted({r, (r + 1) % nv, (r - 1) % nv}) for r in range(nv)]
    ci = np.array([c for row in cols for c in row], np.int32)
    rp = np.concatenate([[0], np.cumsum([len(row) for row in cols])]).astype(np.int32)
    vals = np.zeros((len(ci), 3, 3))
    for r in range(nv):
        for k in range(rp[r], rp[r + 1]):
            vals[k] = 4 * np.eye(3) if ci[k] == r else -0.5 * np.eye(3)
    return rp, ci, vals, np.ones(3 * nv)


@pytest.mark.parametrize("fault", ["missing_diagonal", "duplicate_diagonal", "column_out_of_range", "decreasing_row_pointer"])
def test_pcg_bsr_rejects_malformed_structure(fault):
    """The stand-alone PCG refuses a malformed block-CSR matrix with an
    invalid-argument code before it touches the device."""
    rp, ci, vals, b = _small_block_system()
    ci = ci.copy()
    rp = rp.copy()
    row = list(ci[rp[2]:rp[3]])
    if fault == "missing_diagonal":
        ci[rp[2] + row.index(2)] = 0
    elif fault == "duplicate_diagonal":
        ci[rp[2] + [k for k, c in enumerate(row) if c != 2][0]] = 2
    elif fault == "column_out_of_range":
        ci[4] = 6
    else:
        rp[3] = rp[2] - 1
    with pytest.raises(cipc.CipcError) as e:
        cipc.pcg_bsr(rp, ci, vals, b)
    assert e.value.code == 1
