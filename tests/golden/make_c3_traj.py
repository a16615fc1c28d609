"""Generates tests/golden/c3_traj.npz: trajectories of the large single-run
workload (L=2896, N1=N2=2^20, TSC 2048^2, lambda=256, dt=5e-5) computed by
the reference itself, 1000 steps twice from one non-overlapping start:

  traj       identical injected noise: the Philox uniform-disk stream of key 99
             (the uniforms the CUDA library's BD_NOISE_DISK draws, injected into
             the reference's own noise routine, dynamik_methoden.cpp:1317-1339)
  noiseless  injected u = 0.5, i.e. xi = 0

The compiled reference checker (oracle/_ref/c3/bdref, built from the
reference's sources by oracle/build_ref.py) runs zeitschritt()
(dynamik_methoden.cpp:74-163) with its TSC grid routines
(gridRoutinen.cpp:412-668) and lazy re-binning (:216-325), about 5 s per step
on one core, so the two runs take about 1.5 h in parallel.

The start is bench.start_positions(c3, 31): seeded uniform positions with
pairs closer than 0.8 sigma re-drawn; the fixture keeps a digest of it so a
test can check that it regenerated the same start. To keep the fixture small
it stores every 256th particle of the combined index (species 1 first) at
steps 100, 500 and 1000: cell (git) and offset (rel), and the simulated time.

    python tests/golden/make_c3_traj.py [workdir]
"""
import hashlib
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
import configs as C  # noqa: E402
import oracle as O  # noqa: E402

NAME = "c3"
START_SEED = 31
NOISE_KEY = 99
STEPS = 1000
CKPTS = (100, 500, 1000)
STRIDE = 256


def start(p):
    import bench
    return bench.start_positions(p, START_SEED)


def digest(pos):
    h = hashlib.sha256()
    for s in (0, 1):
        h.update(np.ascontiguousarray(pos[s][0], np.int32).tobytes())
        h.update(np.ascontiguousarray(pos[s][1], np.float64).tobytes())
    return h.hexdigest()


def read_ckpts(path, n_total):
    m = (n_total + STRIDE - 1) // STRIDE
    rec = 4 + 8 + m * 24
    buf = open(path, "rb").read()
    out = []
    for off in range(0, len(buf) - rec + 1, rec):
        st = int(np.frombuffer(buf, np.int32, 1, off)[0])
        t = float(np.frombuffer(buf, np.float64, 1, off + 4)[0])
        a = np.frombuffer(buf[off + 12:off + rec], dtype=[("g", "<i4", 2), ("r", "<f8", 2)])
        out.append((st, t, a["g"].copy(), a["r"].copy()))
    return out


def main():
    work = os.path.abspath(sys.argv[1]) if len(sys.argv) > 1 else os.path.join(ROOT, "_work", "c3_traj")
    os.makedirs(work, exist_ok=True)
    if not O.have_ref(NAME):
        raise SystemExit("reference checker for c3 not built: python oracle/build_ref.py c3")
    p = C.CONFIGS[NAME]
    pos = start(p)
    O.write_pos(os.path.join(work, "start.pos"), pos)
    t0 = time.time()
    procs = {}
    for tag, key in (("traj", str(NOISE_KEY)), ("noiseless", "zero")):
        procs[tag] = subprocess.Popen(
            [O.ref_exe(NAME), "stepsphilox", os.path.join(work, "start.pos"), str(STEPS), key,
             str(STRIDE), ",".join(str(c) for c in CKPTS), os.path.join(work, tag + ".bin")],
            cwd=work, stdout=open(os.path.join(work, tag + ".log"), "w"), stderr=subprocess.STDOUT)
    for tag, q in procs.items():
        if q.wait() != 0:
            raise SystemExit("reference run %s failed (see %s.log)" % (tag, tag))
    n = p["N1"] + p["N2"]
    out = {"start_sha256": np.array(digest(pos)), "start_seed": np.array(START_SEED),
           "noise_key": np.array(NOISE_KEY), "stride": np.array(STRIDE),
           "ckpts": np.array(CKPTS, np.int32)}
    for tag in ("traj", "noiseless"):
        recs = read_ckpts(os.path.join(work, tag + ".bin"), n)
        assert [r[0] for r in recs] == list(CKPTS), [r[0] for r in recs]
        for k, (st, t, g, r) in enumerate(recs):
            out["%s%d_git" % (tag, k)] = g
            out["%s%d_rel" % (tag, k)] = r
            out["%s%d_t" % (tag, k)] = np.array(t)
    np.savez_compressed(os.path.join(HERE, "c3_traj.npz"), **out)
    print("c3_traj.npz written after %.0f s" % (time.time() - t0))


if __name__ == "__main__":
    main()
