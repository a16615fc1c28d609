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


# Largest relative error of the mesh force against the continuum K1 law at
# 3 <= r <= 20 (lam = 5, mesh spacing 0.39): the finite-difference gradient
# and the discrete Laplacian in the Green's function (dynamik_methoden.cpp:
# 1384-1394) give ~1 % at r = 3 for CIC/TSC; NGP's piecewise-constant
# assignment adds a position-dependent error of up to ~5 %.
K1_TOL = {0: 0.08, 1: 0.02, 2: 0.02}


def k1_pair_case(base, scheme, r, ang, species=(0, 0), lam=5.0, gamma=2 * np.pi, f2=0.6,
                 L=100.0, Z=256):
    """Two isolated particles at distance r, direction angle ang from +y, on a
    Z² mesh of spacing L/Z << lam: the krafttestmode set-up (main.cpp:220-248),
    one particle per species given in `species`. Returns (params, positions,
    expected capillary force on the second particle).

    The screened Green's function gamma/(k² + 1/lam²) (dynamik_methoden.cpp:
    1384-1394, 529-613) is gamma/(2π)·K0(r/lam) in the plane, so the pair
    force is attractive with magnitude w_a·w_b·gamma/(2π)·K1(r/lam)/lam, the
    weights being 1 for species 1 and f2_f1 for species 2
    (gridRoutinen.cpp:31-668)."""
    from scipy.special import k1
    import configs as C
    n = [species.count(0), species.count(1)]
    p = dict(C.CONFIGS[base], N1=n[0], N2=n[1], L=L, FFT_samples=Z, densGrid_Schema=scheme,
             lambda_kapillar=lam, kapillar_vorfaktor=gamma, f2_f1=f2)
    B = C.derived(p)["nachList_Breite"]
    u = np.array([np.sin(ang), np.cos(ang)])
    x = np.array([[L / 2 + 0.13, L / 2 + 0.31], [L / 2 + 0.13 + r * u[0], L / 2 + 0.31 + r * u[1]]])
    git = np.floor(x / B).astype(np.int32)
    rel = x - git * B
    pos = {}
    for s in (0, 1):
        idx = [i for i in (0, 1) if species[i] == s]
        pos[s] = (git[idx].reshape(-1, 2), rel[idx].reshape(-1, 2))
    w = [1.0 if s == 0 else f2 for s in species]
    expect = -w[0] * w[1] * gamma / (2 * np.pi) * k1(r / lam) / lam * u
    return p, pos, expect


def pair_forces(f, species):
    """Capillary forces on the two particles of k1_pair_case, in its order."""
    if species[0] == species[1]:
        return f[("kap", species[0])][0], f[("kap", species[0])][1]
    return f[("kap", species[0])][0], f[("kap", species[1])][0]
