"""Resumable binary snapshot: a run stopped, saved, loaded into a fresh
context and stepped on gives the same bits as the uninterrupted run (fused
step, stage kernels with an adaptive dt, radix-3 mesh)."""
import numpy as np
import pytest

import configs as C

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c1_cic", "tiny_tsc", "tiny_cic"])
def test_snapshot_resume_is_bit_identical(gpu, tmp_path, name):
    p = dict(C.CONFIGS[name], noise_kind=gpu.NOISE_GAUSS)
    path = tmp_path / "run.bdsnap"
    a = gpu.Run(p, seed=5)
    a.init_positions(p["startpos_methode"])
    a.zeitschritte(60)
    b = gpu.Run(p, seed=5)
    b.init_positions(p["startpos_methode"])
    b.zeitschritte(25)
    b.snapshot_save(path)
    b.close()
    c = gpu.Run(p, seed=5)
    c.snapshot_load(path)
    assert c.step_count() == 25
    c.zeitschritte(35)
    pa, pc = a.get_positions(), c.get_positions()
    for s in (0, 1):
        assert np.array_equal(pa[s][0], pc[s][0]) and np.array_equal(pa[s][1], pc[s][1])
    assert a.time() == c.time() and a.step_count() == c.step_count() == 60


def test_snapshot_rejects_another_run(gpu, tmp_path):
    p = dict(C.CONFIGS["tiny_cic"])
    path = tmp_path / "run.bdsnap"
    a = gpu.Run(p, seed=5)
    a.init_positions(1)
    a.snapshot_save(path)
    with pytest.raises(gpu.BdError) as e:
        gpu.Run(p, seed=6).snapshot_load(path)  # another noise key
    assert e.value.status == -1
    with pytest.raises(gpu.BdError) as e:
        gpu.Run(dict(p, T=2.0), seed=5).snapshot_load(path)
    assert e.value.status == -1
    (tmp_path / "bad").write_bytes(b"not a snapshot")
    with pytest.raises(gpu.BdError) as e:
        gpu.Run(p, seed=5).snapshot_load(tmp_path / "bad")
    assert e.value.status == -6


def _write_startpos(path, xs, header=("# header 1", "# header 2"), types=(1, 2)):
    with open(path, "w") as f:
        f.write("\n".join(header) + "\n")
        for s, x in enumerate(xs):
            for i, (a, b) in enumerate(x):
                f.write("%d \t %d \t %.9g \t %.9g\n" % (i, types[s], a, b))


def test_init_pos_aus_datei(gpu, tmp_path):
    """startpos.txt reader (init_pos_aus_datei, dynamik_methoden.cpp:
    1578-1643): two header lines, then "idx TAB type TAB x TAB y" rows,
    species 1 first. Coordinates are read as float (%g into float, :1596)
    and split as git = (int)(x / B), rel = x - git*B (the reference's own
    line computes rel = x - rel*B, :1614-1615, which is not reproduced).
    Rows out of order, of the wrong type, or outside [0, L] are errors."""
    p = dict(C.CONFIGS["tiny_cic"])
    d = C.derived(p)
    B, Cn, L = d["nachList_Breite"], d["nachList_Zellen"], p["L"]
    rng = np.random.default_rng(4)
    xs = [rng.uniform(0, L, (p["N1"], 2)), rng.uniform(0, L, (p["N2"], 2))]
    xs[0][0] = (0.0, L)  # the edges: x = L is a legal coordinate
    f = tmp_path / "startpos.txt"
    _write_startpos(f, xs)
    r = gpu.Run(p, seed=1)
    r._call("bd_init_pos_aus_datei", str(f).encode())
    got = r.get_positions()
    for s in (0, 1):
        x = xs[s].astype(np.float32).astype(np.float64)  # %g read into a float
        git = np.minimum((x / B).astype(np.int32), Cn - 1)
        rel = x - git * B
        assert np.array_equal(got[s][0], git), s
        assert np.allclose(got[s][1], rel, rtol=0, atol=2e-6 * B), s
        back = got[s][0] * B + got[s][1]
        assert np.abs(back - x).max() <= 1e-5, s
    # the same positions then step like positions given through bd_set_positions
    q = gpu.Run(p, seed=1)
    q.set_positions(got)
    r.zeitschritte(20)
    q.zeitschritte(20)
    a, b = r.get_positions(), q.get_positions()
    for s in (0, 1):
        assert np.array_equal(a[s][0], b[s][0]) and np.array_equal(a[s][1], b[s][1])
    # errors: wrong type, rows out of order, coordinate outside [0, L], short
    # file, missing file
    cases = [(dict(types=(2, 2)), -6), (dict(), -4), (dict(header=("# one only",)), -6)]
    bad = [x.copy() for x in xs]
    bad[1][3] = (L + 1.0, 2.0)
    for k, (kw, want) in enumerate(cases):
        g = tmp_path / ("bad%d.txt" % k)
        _write_startpos(g, bad if want == -4 else xs, **kw)
        with pytest.raises(gpu.BdError) as e:
            gpu.Run(p, seed=1)._call("bd_init_pos_aus_datei", str(g).encode())
        assert e.value.status == want, (k, e.value.status)
    lines = f.read_text().splitlines()
    (tmp_path / "swap.txt").write_text("\n".join(lines[:2] + [lines[3], lines[2]] + lines[4:]) + "\n")
    with pytest.raises(gpu.BdError) as e:
        gpu.Run(p, seed=1)._call("bd_init_pos_aus_datei", str(tmp_path / "swap.txt").encode())
    assert e.value.status == -6
    with pytest.raises(gpu.BdError) as e:
        gpu.Run(p, seed=1)._call("bd_init_pos_aus_datei", str(tmp_path / "missing.txt").encode())
    assert e.value.status == -6


@pytest.mark.gpu
@pytest.mark.parametrize("n1,n2", [(40000, 30000), (70000, 0)])
def test_positions_round_trip_large(gpu, n1, n2):
    """bd_set_positions_all / bd_get_positions_all on runs large enough for
    the host threads of the conversion: what is read back is what was set
    (offsets rounded to FP32), before and after the cell sort; a position out
    of range anywhere in the arrays is refused with BD_ERR_RANGE and leaves
    the run as it was."""
    import math
    L = math.sqrt(2 * max(n1 + n2, 1) * math.pi / (4 * 0.2))
    p = dict(C.CONFIGS["c1_cic"], N1=n1, N2=n2, L=L, FFT_samples=256, lambda_kapillar=L / 8)
    d = C.derived(p)
    Cc, B = d["nachList_Zellen"], d["nachList_Breite"]
    rng = np.random.default_rng(5)
    pos = {}
    for s, n in ((0, n1), (1, n2)):
        git = rng.integers(0, Cc, (n, 2)).astype(np.int32)
        rel = rng.uniform(0, B, (n, 2))
        pos[s] = (git, rel)
    r = gpu.Run(p, seed=3)
    r.set_positions_all(pos)
    got = r.get_positions()
    for s, n in ((0, n1), (1, n2)):
        assert np.array_equal(got[s][0], pos[s][0])
        assert np.array_equal(got[s][1], pos[s][1].astype(np.float32).astype(np.float64))
    bad = {s: (pos[s][0].copy(), pos[s][1].copy()) for s in (0, 1)}
    s_bad = 1 if n2 else 0
    k = (n2 if n2 else n1) * 3 // 4
    bad[s_bad][0][k, 1] = Cc  # one cell index past the last
    with pytest.raises(gpu.BdError) as ei:
        r.set_positions_all(bad)
    assert ei.value.status == -4  # BD_ERR_RANGE
    after = r.get_positions()
    for s in (0, 1):
        assert np.array_equal(after[s][0], got[s][0]) and np.array_equal(after[s][1], got[s][1])
    r.close()
