"""Local densities of the offline analysis (main_auswertung.cpp:182-390) on
the device, through the C ABI, against the oracle (oracle/bd_oracle.c,
pinned against the reference's own analysis program by
tests/test_oracle.py) on the same FP64 positions.

Tolerances: the device sums each cell with FP64 atomic adds in whatever
order they land, the oracle in particle order, so each cell agrees to 1e-13
of its own value (a few ulp; cells that hold only the far tail of a TSC
weight, around 1e-19, included: the reference counts them in the
|rho1 - rho2| / rho thresholds); histogram and threshold counts agree
exactly except for cells whose value lies within 1e-9 of a bin edge or
threshold, which may fall either way (the test counts those and allows one
move per such cell)."""
import os

import numpy as np
import pytest

import configs as C
from conftest import abs_pos, golden, gpos

pytestmark = pytest.mark.gpu
EDGE = 1e-9


def _oracle(oracle_mod, L, pos, B, lp):
    x = abs_pos(pos, B)
    g1, g2 = oracle_mod.lokale_dichte(L, x[0], x[1], lp.snapgrid_crude)
    hist, over = oracle_mod.rhohist(g1, g2, lp.rhohist_bins, lp.rhohist_drho, list(lp.rho_thresh),
                                    list(lp.drho_thresh))
    return g1, g2, hist, over


def _ambiguous(g1, g2, lp):
    """Cells within EDGE of a bin edge or a threshold, per histogram and for
    the threshold counts."""
    rho, drho = g1 + g2, g1 - g2
    bins = lp.rhohist_bins
    amb = []
    for v in (g1 / lp.rhohist_drho - 0.5, g2 / lp.rhohist_drho - 0.5, rho / lp.rhohist_drho - 0.5,
              drho / lp.rhohist_drho - 0.5 + bins // 2):
        amb.append(int((np.abs(v - np.rint(v)) < EDGE * np.maximum(1.0, np.abs(v))).sum()))
    with np.errstate(invalid="ignore", divide="ignore"):
        q = np.abs(drho) / rho
    t = sum(int((np.abs(rho - th) < EDGE).sum()) for th in lp.rho_thresh)
    t += sum(int((np.abs(q - th) < EDGE).sum()) for th in lp.drho_thresh)
    return amb, t


def _compare(dev, orc, lp, label):
    g1, g2, hist, over = dev
    o1, o2, ohist, oover = orc
    err = max((np.abs(g1 - o1) / np.maximum(np.abs(o1), 1e-300)).max(),
              (np.abs(g2 - o2) / np.maximum(np.abs(o2), 1e-300)).max())
    assert np.array_equal(g1 == 0, o1 == 0) and np.array_equal(g2 == 0, o2 == 0)
    amb, tamb = _ambiguous(o1, o2, lp)
    dh = [int(np.abs(hist[i] - ohist[i]).sum()) for i in range(4)]
    do = int(np.abs(over - oover).sum())
    print("%s: grid max per-cell rel diff %.2e, histogram moves %s (edge cells %s), threshold diff %d (edge %d)"
          % (label, err, dh, amb, do, tamb))
    assert err <= 1e-13
    for i in range(4):
        assert dh[i] <= 2 * amb[i]
        assert hist[i].sum() == g1.size
    assert do <= tamb


@pytest.mark.parametrize("name", ["tiny_cic", "tiny_tsc", "tiny_radial", "c1_cic"])
def test_lokale_dichte_matches_oracle(gpu, oracle_mod, name):
    p = C.CONFIGS[name]
    g = golden(name)
    r = gpu.Run(p, seed=1)
    lp = gpu.lokdens_params()
    for pre in ("init", "start"):
        r.set_positions(gpos(g, pre))
        pos = r.get_positions()
        dev = r.lokale_dichte(lp)
        _compare(dev, _oracle(oracle_mod, p["L"], pos, r.B, lp), lp, "%s %s" % (name, pre))
        again = r.lokale_dichte(lp)
        np.testing.assert_allclose(again[0], dev[0], rtol=1e-13, atol=0)
        np.testing.assert_allclose(again[1], dev[1], rtol=1e-13, atol=0)
    r.close()


def test_lokale_dichte_other_parameters(gpu, oracle_mod):
    """A coarser lattice, other bins and thresholds, after device steps."""
    p = C.CONFIGS["c1_cic"]
    r = gpu.Run(p, seed=4)
    r.set_positions(gpos(golden("c1_cic"), "start"))
    r.zeitschritte(200)
    lp = gpu.lokdens_params(snapgrid_crude=1.7, rhohist_bins=37, rhohist_drho=0.02,
                            rho_thresh=(0.05, 0.3, 0.9), drho_thresh=(0.05, 0.3, 0.7, 0.999))
    pos = r.get_positions()
    _compare(r.lokale_dichte(lp), _oracle(oracle_mod, p["L"], pos, r.B, lp), lp, "c1_cic coarse")
    r.close()


def test_lokale_dichte_medium_full_size(gpu, oracle_mod):
    """The medium single-run workload (L=512, 2 x 32768 particles): 1024^2
    lattice, every cell against the oracle, and the sizes' own properties:
    each species' density integrates to its particle count and each
    histogram holds every cell once."""
    p = C.CONFIGS["c2"]
    r = gpu.Run(p, seed=11)
    r.init_positions(1)
    lp = gpu.lokdens_params()
    dev = r.lokale_dichte(lp)
    pos = r.get_positions()
    _compare(dev, _oracle(oracle_mod, p["L"], pos, r.B, lp), lp, "c2 full size")
    n = dev[0].shape[0]
    w = p["L"] / n
    assert n == 1024
    assert abs(dev[0].sum() * w * w - p["N1"]) <= 1e-9 * p["N1"]
    assert abs(dev[1].sum() * w * w - p["N2"]) <= 1e-9 * p["N2"]
    r.close()


HEADERS = {
    "rhoHist.txt": ["# Format: t TAB dens TAB fraction of space with <rho1 TAB rho2 TAB rho1+rho2> = dens "],
    "drhoHist.txt": ["# Format: t TAB rho1-rho2 TAB fraction of space with this rho1-rho2"],
    "rhoThresh.txt": ["# Format: t TAB #cells over thresh1 TAB #cells over thresh2 TAB #cells over thresh3",
                      "# where thresh1=0.1, thresh2=0.2, thresh3=0.5"],
    "drhoThresh.txt": ["# Format: t TAB #cells with |rho1-rho2|/(rho1+rho2) over thresh1 TAB same thresh2 TAB "
                       "same thresh3 TAB same thresh4",
                       "# where thresh1=0.1, thresh2=0.2, thresh3=0.5, thresh4=0.99"],
}


def _frames(path):
    frames, cur = [], []
    for line in open(path):
        s = line.strip()
        if s.startswith("#"):
            continue
        if not s:
            if cur:
                frames.append(np.array(cur))
                cur = []
            continue
        cur.append([float(v) for v in s.split(" \t ")])
    if cur:
        frames.append(np.array(cur))
    return frames


def test_schreibe_lokale_dichte_files(gpu, tmp_path):
    """The analysis program's files (main_auswertung.cpp:60-77,205-210,
    290-296,357-375): headers, one block per frame, the printed values of
    the device results."""
    p = C.CONFIGS["tiny_cic"]
    r = gpu.Run(p, seed=2)
    r.set_positions(gpos(golden("tiny_cic"), "start"))
    res = []
    for nr in range(3):
        r.schreibe_lokale_dichte(tmp_path, nr)
        res.append(r.lokale_dichte())
        r.zeitschritte(50)
    r.close()
    for f, hdr in HEADERS.items():
        lines = open(tmp_path / f).read().split("\n")
        assert lines[:len(hdr)] == hdr and lines[len(hdr)] == ""
    n = res[0][0].shape[0]
    pref = 1.0 / (n * n)
    rh, dh = _frames(tmp_path / "rhoHist.txt"), _frames(tmp_path / "drhoHist.txt")
    rt, dt = _frames(tmp_path / "rhoThresh.txt")[0], _frames(tmp_path / "drhoThresh.txt")[0]
    assert len(rh) == len(dh) == 3 and rt.shape == (3, 4) and dt.shape == (3, 5)
    for nr, (g1, g2, hist, over) in enumerate(res):
        t = nr * p["obs_dt"]
        loc = open(tmp_path / "localDens" / ("rho%d.txt" % nr)).read().split("\n")
        assert loc[:3] == ["# Format: t x y rho1 rho2 ", "# where x and y are the center of the cell. ", ""]
        grid = _frames(tmp_path / "localDens" / ("rho%d.txt" % nr))
        assert len(grid) == 1 and grid[0].shape == (n * n, 5)
        w = p["L"] / n
        k, l = np.divmod(np.arange(n * n), n)
        np.testing.assert_allclose(grid[0][:, 0], t, rtol=1e-5)
        np.testing.assert_allclose(grid[0][:, 1], (k + 0.5) * w, rtol=6e-6)
        np.testing.assert_allclose(grid[0][:, 2], (l + 0.5) * w, rtol=6e-6)
        np.testing.assert_allclose(grid[0][:, 3], g1.ravel(), rtol=6e-6, atol=1e-300)
        np.testing.assert_allclose(grid[0][:, 4], g2.ravel(), rtol=6e-6, atol=1e-300)
        bins = hist.shape[1]
        np.testing.assert_allclose(rh[nr][:, 1], 0.01 * (np.arange(bins) + 0.5), rtol=6e-6)
        np.testing.assert_allclose(rh[nr][:, 2:], (hist[[0, 1, 2]] * pref).T, rtol=6e-6)
        np.testing.assert_allclose(dh[nr][:, 1], 0.01 * (np.arange(bins) + 0.5 - bins // 2), rtol=6e-6)
        np.testing.assert_allclose(dh[nr][:, 2], hist[3] * pref, rtol=6e-6)
        np.testing.assert_allclose(rt[nr, 1:], over[:3] * pref, rtol=6e-6)
        np.testing.assert_allclose(dt[nr, 1:], over[3:] * pref, rtol=6e-6)


def test_lokale_dichte_rejects_bad_parameters(gpu):
    r = gpu.Run(C.CONFIGS["tiny_cic"], seed=1)
    r.set_positions(gpos(golden("tiny_cic"), "init"))
    for kw in (dict(snapgrid_crude=0.0), dict(rhohist_bins=0), dict(rhohist_drho=0.0)):
        with pytest.raises(gpu.BdError):
            r.lokale_dichte(gpu.lokdens_params(**kw))
    with pytest.raises(gpu.BdError):
        r.lokale_dichte(gpu.lokdens_params(rhohist_bins=4096))
    r.close()
