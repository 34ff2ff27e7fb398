import importlib
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle")
for p in (ROOT, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    # the CPU checker is test infrastructure; build it if a fresh checkout lacks it
    if not os.path.exists(os.path.join(ORACLE, "liboracle.so")):
        subprocess.call(["make", "-s", "-C", ORACLE, "liboracle.so"])
    import __graft_entry__

    ref = __graft_entry__.REFERENCE
    if (not os.path.exists(os.path.join(ORACLE, "_ref", "libim3d_ref.so"))
            and os.path.isdir(os.path.join(ref, "header"))):
        subprocess.call(["make", "-s", "-C", ORACLE, "ref", f"REF={ref}"])


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module("3dimagetoolkit_b200")


@pytest.fixture(scope="session")
def O():
    import oracle_py

    return oracle_py


@pytest.fixture(scope="session")
def ctx(pkg):
    c = pkg.Context(0)
    yield c
    c.close()


def rel(a, b):
    import numpy as np

    # complex arrays (the FFT checks) keep their imaginary parts
    dt = np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64
    a = np.asarray(a, dtype=dt)
    b = np.asarray(b, dtype=dt)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
