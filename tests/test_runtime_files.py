"""The headless runner's runtime files in the reference's formats, no GPU:
checkpoint positions and inertial target (mesh3D::output_tetTempData /
load_tetTempData, SimulationMesh.cpp:470-543), checkpoint totals and the
per-step timeCost.txt summary (IPCSolver.cpp:1085-1101, 1261-1273,
1318-1332).  The files are compared byte for byte with text written here by
the formatting rules the reference's streams follow (17 significant digits
for positions, the default six for the totals)."""
import ctypes as C
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
APPS = os.path.join(HERE, "..", "cpu-ipc_b200", "apps")
dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)


@pytest.fixture(scope="module")
def rf():
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("g++ not available")
    d = tempfile.mkdtemp()
    so = os.path.join(d, "librf.so")
    subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-I", APPS, "-o", so,
                    os.path.join(HERE, "runtime_files_harness.cpp")], check=True)
    L = C.CDLL(so)
    L.rf_write_state.argtypes = [C.c_char_p, dp, dp, C.c_int]
    L.rf_load_state.argtypes = [C.c_char_p, C.c_int, dp, dp]
    L.rf_write_totals.argtypes = [C.c_char_p, dp, C.c_double, C.c_longlong, C.c_int, C.c_double]
    L.rf_load_totals.argtypes = [C.c_char_p, dp, dp, C.POINTER(C.c_longlong), ip, dp]
    L.rf_write_summary.argtypes = [C.c_char_p, dp, C.c_double, C.c_longlong, C.c_int, C.c_double]
    return L


def _p(a):
    return a.ctypes.data_as(dp)


def _state(rng, nv):
    x = rng.standard_normal((nv, 3)) * 10.0 ** rng.integers(-6, 4, (nv, 1))
    x[0] = [0.25, -1.0, 0.0]
    x[1] = [1e-300, 123456789.0, -0.1]
    return x


def test_checkpoint_positions_are_written_in_the_reference_format(rf, tmp_path):
    rng = np.random.default_rng(3)
    x, xt = _state(rng, 7), _state(rng, 7)
    out = str(tmp_path / "run")
    assert rf.rf_write_state(out.encode(), _p(x), _p(xt), 7) == 1
    for name, a in (("vertex.txt", x), ("vertexXtile.txt", xt)):
        text = open(os.path.join(out, "tempData", name)).read()
        assert text == "".join("%.17g %.17g %.17g\n" % tuple(r) for r in a)


def test_checkpoint_positions_round_trip_and_reject_another_mesh(rf, tmp_path):
    rng = np.random.default_rng(4)
    x, xt = _state(rng, 9), _state(rng, 9)
    out = str(tmp_path / "run").encode()
    rf.rf_write_state(out, _p(x), _p(xt), 9)
    a, b = np.zeros((9, 3)), np.zeros((9, 3))
    assert rf.rf_load_state(out, 9, _p(a), _p(b)) == 1
    assert np.array_equal(a, x) and np.array_equal(b, xt)
    z = np.zeros((12, 3))
    assert rf.rf_load_state(out, 10, _p(z), _p(z)) == 0  # too few vertices
    assert rf.rf_load_state(out, 8, _p(z), _p(z)) == 0   # data left over
    assert rf.rf_load_state(str(tmp_path / "none").encode(), 9, _p(z), _p(z)) == 0


def test_checkpoint_written_by_the_reference_layout_loads(rf, tmp_path):
    # the reference's own writer: one "x y z" line per vertex, std::endl
    d = tmp_path / "ref" / "tempData"
    d.mkdir(parents=True)
    x = np.arange(12, dtype=float).reshape(4, 3) / 7.0
    (d / "vertex.txt").write_text("".join("%.17g %.17g %.17g\n" % tuple(r) for r in x))
    (d / "vertexXtile.txt").write_text("".join("%.17g %.17g %.17g\n" % tuple(r) for r in -x))
    a, b = np.zeros((4, 3)), np.zeros((4, 3))
    assert rf.rf_load_state(str(tmp_path / "ref").encode(), 4, _p(a), _p(b)) == 1
    assert np.array_equal(a, x) and np.array_equal(b, -x)
    (d / "vertex.txt").write_text("0 0 0\n1 1 nan_or_text\n")
    assert rf.rf_load_state(str(tmp_path / "ref").encode(), 2, _p(a), _p(b)) == 0


def test_checkpoint_totals_format_and_round_trip(rf, tmp_path):
    stage = np.array([1234.5678901, 0.000123456789, 98765432.1, 5.0, 0.0])
    out = str(tmp_path / "run").encode()
    assert rf.rf_write_totals(out, _p(stage), 3.14159265358979, 4321, 40, 123456.789) == 1
    text = open(os.path.join(tmp_path, "run", "tempData", "timeCost.txt")).read()
    want = "".join("%g\n" % v for v in stage) + "%g\n" % 3.14159265358979 + "4321\n40\n" + "%g\n" % 123456.789
    assert text == want
    s5, sm, kp = np.zeros(5), C.c_double(), C.c_double()
    nw, si = C.c_longlong(), C.c_int()
    assert rf.rf_load_totals(out, _p(s5), C.byref(sm), C.byref(nw), C.byref(si), C.byref(kp)) == 1
    assert nw.value == 4321 and si.value == 40
    # six significant digits survive, as in the reference's resume
    assert abs(kp.value - 123456.789) <= 1e-5 * 123456.789
    assert np.allclose(s5, stage, rtol=1e-5)
    assert rf.rf_load_totals(str(tmp_path / "none").encode(), _p(s5), C.byref(sm), C.byref(nw), C.byref(si), C.byref(kp)) == 0


def test_time_summary_lines(rf, tmp_path):
    stage = np.array([1500.0, 2500.0, 10.0, 20.0, 0.5])
    out = str(tmp_path / "run")
    assert rf.rf_write_summary(out.encode(), _p(stage), 4600.0, 30, 12, 451.0) == 1
    text = open(os.path.join(out, "timeCost.txt")).read()
    want = "".join("time%d: %g\n" % (k, stage[k] / 1000.0) for k in range(5))
    want += "timeAll: %g\ntotal iter: 30\nframes: 12\ntotalCollisionNum: %g\naverageCollision: %g\n" % (4.6, 451.0, 451.0 / 30)
    assert text == want
