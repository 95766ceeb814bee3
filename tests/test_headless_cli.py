"""The headless runner's command line (cpu-ipc_b200/cipc_headless_gpu), no
GPU: options are parsed and scenes are built before the first library call,
so usage, bad values and missing inputs are reported as the reference's
runner reports them (a message and exit status 1; apps/cipc_headless.cpp)."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
EXE = os.path.join(HERE, "..", "cpu-ipc_b200", "cipc_headless_gpu")


def _run(*args):
    if not os.path.exists(EXE):
        pytest.skip("headless runner not built")
    return subprocess.run([EXE, *args], capture_output=True, text=True, timeout=60)


def test_help_lists_the_options():
    r = _run("--help")
    assert r.returncode == 0
    for opt in ("--scene", "--steps", "--output", "--resume", "--write-checkpoints", "--hinge-bending",
                "--precision", "--precond", "--linear-solver", "--no-output"):
        assert opt in r.stdout, opt
    assert "bunny2" in r.stdout


@pytest.mark.parametrize("args,message", [
    (("--bogus",), "unknown option: --bogus"),
    (("--steps", "-2"), "--steps expects a non-negative integer"),
    (("--steps",), "--steps requires a value"),
    (("--precision", "fp16"), "unknown precision: fp16"),
    (("--precond", "ilu"), "unknown preconditioner: ilu"),
    (("--linear-solver", "pardiso"), "is not part of this build"),
    (("--scene", "bunny2"), "needs --assets"),
    (("--scene", "cloth-bunny", "--assets", "/nonexistent"), "cannot open /nonexistent/scene/parameterSetting.txt"),
    (("--scene", "teapot"), "unknown scene: teapot"),
])
def test_bad_input_is_reported(args, message):
    r = _run(*args)
    assert r.returncode == 1
    assert message in r.stderr
