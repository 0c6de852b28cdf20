import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "nanoj-esrrf_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def golden_names(kind=None):
    names = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))
    if kind:
        names = [n for n in names if n.startswith(kind + "_")]
    return names


def rel_err(a, b):
    """Max abs difference over the reference output's dynamic range, per slice."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    rng = b.max() - b.min()
    return float(np.abs(a - b).max() / (rng if rng > 0 else 1.0))


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def esrrf_mod():
    import esrrf
    esrrf.lib()
    return esrrf
