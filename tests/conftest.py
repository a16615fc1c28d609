import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "bd-simulations_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def bdsim_mod():
    import bdsim
    if not os.path.exists(bdsim.LIB_PATH):
        sys.path.insert(0, os.path.join(ROOT, "bd-simulations_b200"))
        import build as bdbuild
        bdbuild.build()
    return bdsim


@pytest.fixture(scope="session")
def gpu(bdsim_mod):
    n = bdsim_mod.device_count()
    assert n > 0, "no CUDA device visible"
    return bdsim_mod


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def gpos(g, prefix):
    return {s: (g["%s_git%d" % (prefix, s)], g["%s_rel%d" % (prefix, s)]) for s in (0, 1)}


def rel_l2(a, b):
    a = np.concatenate([np.asarray(x).ravel() for x in a])
    b = np.concatenate([np.asarray(x).ravel() for x in b])
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def abs_pos(pos, B):
    return {s: pos[s][0] * B + pos[s][1] for s in (0, 1)}


def min_image(d, L):
    return d - L * np.round(d / L)
