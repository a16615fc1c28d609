"""Generates tests/golden/obs.npz: the reference's own in-run observables,
record_korrelationsfunktion11/12/22 (auswertung.cpp:110-188) and
record_ftrho_unkorrigiert with its |q|^2 binning (init_ftrho, auswertung.cpp:
262-375), computed by the compiled reference checker (oracle/_ref/<config>/
bdref, built by oracle/build_ref.py) on two position sets per configuration:

  a  the reference's init_zufallspos positions of seed 7 (the "init" set of
     <config>.npz), offsets rounded to FP32 (the device keeps FP32 offsets)
  b  the same cells with every species-1 particle at offset (r, r): the
     reference's species-1 rho(k) loop takes y from the x offset
     (auswertung.cpp:333), which then equals the y offset, so the reference's
     species-1 sums can be compared too

Parameters from the generated parameter.h: korr_dr = 0.2, korr_rmax = L/2,
ftrho_qbins = 30, ftrho_dq = 4 pi / L (parameter.h:101-108, 209).

    python tests/golden/make_obs_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

NAMES = ("tiny_cic", "c1_cic")


def position_sets(name):
    g = dict(np.load(os.path.join(HERE, name + ".npz")))
    a = {s: (g["init_git%d" % s].astype(np.int32),
             g["init_rel%d" % s].astype(np.float32).astype(np.float64)) for s in (0, 1)}
    b = dict(a)
    r = a[0][1][:, 0].copy()
    b[0] = (a[0][0], np.stack([r, r], 1))
    return {"a": a, "b": b}


def main():
    out = {}
    for name in NAMES:
        if not O.have_ref(name):
            raise SystemExit("reference checker for %s not built: python oracle/build_ref.py" % name)
        for tag, pos in position_sets(name).items():
            res = O.ref_obs(name, pos)
            for k, v in res.items():
                out["%s_%s_%s" % (name, tag, k)] = v
            for s in (0, 1):
                out["%s_%s_git%d" % (name, tag, s)] = pos[s][0]
                out["%s_%s_rel%d" % (name, tag, s)] = pos[s][1]
    np.savez_compressed(os.path.join(HERE, "obs.npz"), **out)
    print("obs.npz:", len(out), "arrays")


if __name__ == "__main__":
    main()
