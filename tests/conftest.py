"""Shared fixtures.  Tests marked ``gpu`` need a B200 and the built library;
everything else runs on the CPU (oracle, fixtures, ABI surface)."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mtl4-mirror_b200")
sys.path.insert(0, os.path.join(PKG, "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_built():
    lib = os.path.join(PKG, "lib", "libmtlgpu.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", PKG, "-j8"], check=True, capture_output=True)
    orc = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
    if not os.path.exists(orc):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "restatement"], check=True,
                       capture_output=True)


_ensure_built()


@pytest.fixture(scope="session")
def M():
    import mtlgpu
    return mtlgpu


@pytest.fixture(scope="session")
def restate():
    import oracle
    return oracle.Restatement()


@pytest.fixture(scope="session")
def reference():
    """The MTL4 reference compiled from its own headers, when it was built."""
    import oracle
    ref = oracle.available_reference()
    if ref is None:
        pytest.skip("reference build (oracle/_ref) not available")
    return ref


@pytest.fixture(scope="session")
def ctx(M):
    c = M.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def golden():
    path = os.path.join(ROOT, "tests", "golden", "golden.npz")
    return dict(np.load(path, allow_pickle=False))
