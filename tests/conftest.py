"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU.

The oracle (oracle/, test infrastructure only) is the checker: the CUDA path
under test is cl2qcd_b200 (libc2q_b200.so), called through its C ABI.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_oracle():
    import oracle as O
    if not O.available("port"):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return O


@pytest.fixture(scope="session")
def O():
    return _ensure_oracle()


@pytest.fixture(scope="session")
def port(O):
    return O.Oracle("port")


@pytest.fixture(scope="session")
def ref(O):
    if not O.available("reference"):
        pytest.skip("oracle/_ref/libc2q_ref.so (reference kernels) not built here")
    return O.Oracle("reference")


@pytest.fixture(scope="session")
def lib():
    from cl2qcd_b200 import build, _lib
    build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def system(lib):
    import cl2qcd_b200 as c2q
    s = c2q.System(0)
    yield s
    s.close()


def rel_l2(a, b):
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)
