import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "cpu-ipc_b200"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path against the oracle")
    # build the libraries in-tree when a fresh checkout lacks them
    lib = os.path.join(ROOT, "cpu-ipc_b200", "libcipc_gpu.so")
    if not os.path.exists(lib):
        subprocess.run([sys.executable, os.path.join(ROOT, "cpu-ipc_b200", "build.py")], check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    return oracle


@pytest.fixture(scope="session")
def cipc_mod():
    import cipc
    return cipc
