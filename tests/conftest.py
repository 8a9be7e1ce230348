import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def gfk():
    import __graft_entry__
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def engine(gfk):
    eng = gfk.Engine(0)
    yield eng
    eng.close()


def as_tuples(stack):
    return [(l.thickness, l.vp, l.vs, l.density, l.qs, l.qp) for l in stack]


def rel_l2(a, b):
    import numpy as np
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
