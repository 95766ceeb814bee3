"""The library's rest-state set-up (cpu-ipc_b200/csrc/scene_setup.cpp, run by
cipc_gpu_create) built for the host and compared with the oracle's
(initMesh3D, getSurface, the bending set-up and buildModels' scalars,
Simulator.cpp:48-141, 426-529, SimulationMesh.cpp:545-716), no GPU.  The
surface lists must agree entry for entry and in order: their order fixes
edge orientation and hence the contact encodings."""
import ctypes as C
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "..", "cpu-ipc_b200", "csrc")
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
sys.path.insert(0, os.path.join(HERE, "..", "cpu-ipc_b200"))

import cipc  # noqa: E402
import oracle  # noqa: E402
import ref_scenes  # noqa: E402

dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
PARAMS = ("density", "cloth_density", "thickness", "E", "nu", "clothE", "shearE", "bendE", "strainRate", "relDhat")
SCALARS = ("lengthRate", "volumeRate", "stretchS", "shearS", "plateRigidity", "meanMass", "avgEdge", "bboxDiag2",
           "Hhat", "Fhat", "dTol")


@pytest.fixture(scope="module")
def ss():
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("g++ not available")
    d = tempfile.mkdtemp()
    so = os.path.join(d, "libss.so")
    subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-I", SRC, "-o", so,
                    os.path.join(HERE, "scene_setup_harness.cpp"), os.path.join(SRC, "scene_setup.cpp")], check=True)
    L = C.CDLL(so)
    L.ss_setup.restype = C.c_int
    L.ss_setup.argtypes = [C.c_int, dp, C.c_int, ip, C.c_int, ip, dp, dp, C.c_int, dp, dp]
    L.ss_size.restype = C.c_longlong
    L.ss_size.argtypes = [C.c_int]
    L.ss_get.argtypes = [C.c_int, C.c_void_p]
    L.ss_scalars.argtypes = [dp]
    return L


def _setup(L, sc):
    x = np.ascontiguousarray(sc["x"], np.float64).reshape(-1)
    tets = np.ascontiguousarray(sc.get("tets", np.zeros((0, 4))), np.int32).reshape(-1)
    tris = np.ascontiguousarray(sc.get("tris", np.zeros((0, 3))), np.int32).reshape(-1)
    te = sc.get("tetE")
    te = None if te is None else np.ascontiguousarray(te, np.float64)
    p = np.array([float(sc["params"][k]) for k in PARAMS])
    lo, hi = np.array(sc["bbox_min"], np.float64), np.array(sc["bbox_max"], np.float64)
    rc = L.ss_setup(len(x) // 3, x.ctypes.data_as(dp), len(tets) // 4, tets.ctypes.data_as(ip), len(tris) // 3,
                    tris.ctypes.data_as(ip), None if te is None else te.ctypes.data_as(dp), p.ctypes.data_as(dp),
                    int(sc["params"].get("quad_bending", 1)), lo.ctypes.data_as(dp), hi.ctypes.data_as(dp))
    assert rc == 0

    def get(which, dtype):
        n = L.ss_size(which)
        a = np.zeros(n, dtype)
        if n:
            L.ss_get(which, a.ctypes.data_as(C.c_void_p))
        return a
    s = np.zeros(11)
    L.ss_scalars(s.ctypes.data_as(dp))
    return get, dict(zip(SCALARS, s))


# relative to each array's scale: entries that cancel to ~1e-5 of their row
# (the rotated cloth plane of cloth-bunny, whose normal components are ~1e-17)
# differ in their own last digits between the two formula orders
def _close(a, b, rel=1e-12):
    a, b = np.asarray(a, np.float64).reshape(-1), np.asarray(b, np.float64).reshape(-1)
    assert a.shape == b.shape
    if a.size:
        assert np.abs(a - b).max() <= rel * max(np.abs(b).max(), 1e-300)


def _scenes():
    yield "two_cubes", lambda: cipc.scene_two_cubes(3)
    yield "cloth_drape", lambda: cipc.scene_cloth_drape(12, 3)
    yield "pile", lambda: cipc.scene_pile(3, 2, seed=5)
    yield "twist", lambda: cipc.scene_twist(2, 8, 6)
    if ref_scenes.assets_available():
        yield "twisting_mat", lambda: ref_scenes.twisting_mat()
        yield "cloth_bunny", lambda: ref_scenes.cloth_bunny()


@pytest.mark.parametrize("name,make", list(_scenes()))
def test_setup_matches_the_oracle(ss, name, make):
    sc = make()
    get, scal = _setup(ss, sc)
    o = oracle.Oracle(sc)
    faces, verts, edges = o.surface()
    assert np.array_equal(get(21, np.int32), np.asarray(faces).reshape(-1))
    assert np.array_equal(get(22, np.int32), np.asarray(verts).reshape(-1))
    assert np.array_equal(get(23, np.int32), np.asarray(edges).reshape(-1))
    r = o.rest()
    _close(get(1, np.float64), r["DmInv"])
    _close(get(2, np.float64), r["vol"])
    _close(get(3, np.float64), r["DmInv2"])
    _close(get(4, np.float64), r["area"])
    assert np.array_equal(get(20, np.int32), r["bend_v"].reshape(-1))
    _close(get(5, np.float64), r["bend_Q"])
    _close(get(0, np.float64), o.get("mass"))
    os_ = o.scalars()
    for k in SCALARS:
        _close([scal[k]], [os_[k]])
