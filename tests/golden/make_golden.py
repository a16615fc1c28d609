"""Generates the golden fixtures in tests/golden/ from the reference itself.

Runs the compiled reference checker (oracle/_ref/<config>/bdref, built from
the reference's own sources by oracle/build_ref.py) and stores its outputs as
small compressed .npz files, so that tests on machines without the reference
sources can still compare against the reference's own numbers.

    python tests/golden/make_golden.py

Fixtures per configuration (see oracle/configs.py for the parameters):
  init       positions from the reference's init_zufallspos with seed 7
  forces     F?_WCA, F?kap on those positions (+ rho, Fx, Fy for Z <= 128)
  lists      neighbour lists (erwNachbarn) after WCA_init, for tiny_cic
  traj       positions after injected-noise steps from a non-overlapping
             seeded start (Philox uniform-disk noise, key 99), at checkpoints
  noiseless  c1_cic: 1000 steps with injected u = 0.5 (xi = 0)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import configs as C  # noqa: E402
import oracle as O  # noqa: E402

INIT_SEED = 7
START_SEED = 3
NOISE_KEY = 99

TRAJ = {  # config: (steps, checkpoint every)
    "tiny_ngp": (200, 50), "tiny_cic": (200, 50), "tiny_tsc": (200, 50),
    "tiny_radial": (200, 50), "tiny_flags": (200, 50), "tiny_idgas": (200, 50),
    "ref_default": (100, 25), "c1_cic": (1000, 250), "c1_ngp": (200, 100),
    "c1_tsc": (200, 100),
}


def pack_pos(prefix, pos, out):
    for s in (0, 1):
        out["%s_git%d" % (prefix, s)] = pos[s][0].astype(np.int32)
        out["%s_rel%d" % (prefix, s)] = pos[s][1].astype(np.float64)


def philox_uniforms(p, nsteps):
    us = []
    for st in range(nsteps):
        _, u = O.philox_noise(NOISE_KEY, st, p["N1"], p["N2"], gauss=False, with_u=True)
        us.append(u)
    return np.array(us)


def make(name):
    p = C.CONFIGS[name]
    out = {}
    pos = O.ref_init(name, INIT_SEED)
    pack_pos("init", pos, out)
    f = O.ref_forces(name, pos, p["FFT_samples"])
    assert f["oob_messages"] == 0
    for (kind, s) in [("wca", 0), ("wca", 1), ("kap", 0), ("kap", 1)]:
        out["forces_%s%d" % (kind, s)] = f[(kind, s)]
    if p["FFT_samples"] <= 128:
        out["grid_rho"] = f["rho"]
        out["grid_Fx"] = f["Fx"]
        out["grid_Fy"] = f["Fy"]
    if name == "tiny_cic":
        d = C.derived(p)
        lists = O.ref_lists(name, pos, d["nachList_Zellen"])
        for s in (0, 1):
            lens = np.array([len(lists[s][(i, j)]) for i in range(d["nachList_Zellen"])
                             for j in range(d["nachList_Zellen"])], np.int32)
            ids = np.concatenate([lists[s][(i, j)] for i in range(d["nachList_Zellen"])
                                  for j in range(d["nachList_Zellen"])]).astype(np.int32)
            out["lists_len%d" % s] = lens
            out["lists_ids%d" % s] = ids
    steps, every = TRAJ[name]
    if p["startpos_methode"] == 1:
        start = O.nonoverlap_positions(p, START_SEED)
    else:  # deterministic start of the config's own initialiser
        start = pos
    pack_pos("start", start, out)
    u = philox_uniforms(p, steps)
    recs, oob = O.ref_steps(name, start, steps, every, u)
    assert oob == 0
    for k, (t, q) in enumerate(recs):
        pack_pos("traj%d" % k, q, out)
        out["traj%d_t" % k] = np.array(t)
    out["traj_every"] = np.array(every)
    out["traj_steps"] = np.array(steps)
    if name == "c1_cic":
        u0 = np.full((steps, p["N1"] + p["N2"], 2), 0.5)
        recs, oob = O.ref_steps(name, start, steps, every, u0)
        assert oob == 0
        for k, (t, q) in enumerate(recs):
            pack_pos("noiseless%d" % k, q, out)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return name


if __name__ == "__main__":
    names = sys.argv[1:] or list(TRAJ)
    for n in names:
        if not O.have_ref(n):
            raise SystemExit("reference checker for %s not built: python oracle/build_ref.py" % n)
    for n in names:
        print("golden:", make(n))
