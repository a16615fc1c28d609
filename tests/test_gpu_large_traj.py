"""Trajectory parity of the large single-run workload (L=2896, N1=N2=2^20,
TSC 2048^2, lambda=256, dt=5e-5) against the reference itself: 1000 steps
with identical injected noise and 1000 noiseless steps from one
non-overlapping start, compared at steps 100, 500 and 1000 on every 256th
particle (tests/golden/c3_traj.npz, made by tests/golden/make_c3_traj.py
from the compiled reference's zeitschritt, dynamik_methoden.cpp:74-163, with
its TSC grid routines, gridRoutinen.cpp:412-668, and re-binning, :216-325).
"""
import os
import sys

import numpy as np
import pytest

import configs as C
from conftest import GOLDEN, ROOT, min_image

pytestmark = pytest.mark.gpu

# Position error bounds (rms, max over the sampled particles) at each
# checkpoint, about ten times the errors measured on a B200 (after 1000
# steps: injected noise 5.1e-7 rms, 2.5e-6 max; noiseless 9.4e-7 rms,
# 3.6e-5 max; no cell key differs).
TOL = {"traj": (5e-6, 3e-5), "noiseless": (1e-5, 4e-4)}


@pytest.fixture(scope="module")
def c3_case():
    g = dict(np.load(os.path.join(GOLDEN, "c3_traj.npz")))
    sys.path.insert(0, ROOT)
    import bench
    sys.path.insert(0, os.path.join(GOLDEN))
    import make_c3_traj
    p = C.CONFIGS["c3"]
    start = bench.start_positions(p, int(g["start_seed"]))
    assert make_c3_traj.digest(start) == str(g["start_sha256"]), "regenerated start differs from the fixture's"
    return p, g, start


@pytest.mark.parametrize("tag", ["traj", "noiseless"])
def test_large_run_trajectory_vs_reference(gpu, c3_case, tag):
    p, g, start = c3_case
    noise = gpu.NOISE_DISK if tag == "traj" else gpu.NOISE_NONE
    r = gpu.Run(dict(p, noise_kind=noise), seed=int(g["noise_key"]))
    r.set_positions(start)
    r.set_step(0)
    B = C.derived(p)["nachList_Breite"]
    L = p["L"]
    stride = int(g["stride"])
    done = 0
    rows = []
    for k, ck in enumerate(g["ckpts"]):
        r.zeitschritte(int(ck) - done)
        done = int(ck)
        pos = r.get_positions()
        git = np.concatenate([pos[0][0], pos[1][0]])[::stride]
        rel = np.concatenate([pos[0][1], pos[1][1]])[::stride]
        ref_git, ref_rel = g["%s%d_git" % (tag, k)], g["%s%d_rel" % (tag, k)]
        d = min_image((git * B + rel) - (ref_git * B + ref_rel), L)
        rms, mx = float(np.sqrt((d ** 2).mean())), float(np.abs(d).max())
        keys = int(np.any(git != ref_git, axis=1).sum())
        rows.append((int(ck), rms, mx, keys))
        assert abs(r.time() - float(g["%s%d_t" % (tag, k)])) <= 1e-12 * done
    r.close()
    print(tag, ["step %d rms %.2e max %.2e keys differing %d" % row for row in rows])
    tol_rms, tol_max = TOL[tag]
    for step, rms, mx, keys in rows:
        assert rms <= tol_rms and mx <= tol_max, (step, rms, mx)
        assert keys <= len(ref_git) // 2000, (step, keys)
