"""Generates tests/golden/localdens.npz from the reference's own offline
analysis program (main_auswertung.cpp, compiled by
oracle/build_ref.py:build_auswertung from the reference sources).

    python tests/golden/make_localdens_golden.py

For each configuration below, position frames from the step fixtures
(<config>.npz: the reference's init positions and the last trajectory
checkpoint) are written as pos1_1.txt / pos2_1.txt the way
RunObs::schreibe_pos writes them, the analysis program runs on them, and
its outputs are stored per frame f:
  <config>_f<f>_x1, _x2     positions as the program read them (float text)
  <config>_f<f>_g1, _g2     localDens/rho<f>.txt density columns (float32,
                            as printed with %g; only where GRIDS lists it)
  <config>_f<f>_hist        rhoHist / drhoHist counts [4, bins]
                            (rho1, rho2, rho1+rho2, rho1-rho2)
  <config>_f<f>_over        rhoThresh / drhoThresh counts [7]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import build_ref  # noqa: E402
import oracle as O  # noqa: E402

CONFIGS = ["tiny_cic", "tiny_tsc", "tiny_radial", "c1_cic"]
GRIDS = {"tiny_cic", "tiny_tsc", "tiny_radial"}


def _frames(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    last = max(int(k[4:].split("_")[0]) for k in z.files if k.startswith("traj") and k.endswith("_git0"))
    pos = lambda pre: {s: (z["%s_git%d" % (pre, s)], z["%s_rel%d" % (pre, s)]) for s in (0, 1)}
    return [pos("init"), pos("traj%d" % last)]


def main():
    out = {}
    for name in CONFIGS:
        frames = _frames(name)
        build_ref.build_auswertung(name, len(frames))
        for f, r in enumerate(O.ref_auswertung(name, frames)):
            key = "%s_f%d_" % (name, f)
            out[key + "x1"] = r["x1"].astype(np.float32)
            out[key + "x2"] = r["x2"].astype(np.float32)
            if name in GRIDS:
                out[key + "g1"] = r["g1"].astype(np.float32)
                out[key + "g2"] = r["g2"].astype(np.float32)
            out[key + "hist"] = r["hist"]
            out[key + "over"] = r["over"]
        print("localdens golden:", name)
    np.savez_compressed(os.path.join(HERE, "localdens.npz"), **out)


if __name__ == "__main__":
    main()
