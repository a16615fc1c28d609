"""Observables computed on the device from the resident state: g11/g12/g22
(record_korrelationsfunktion*) and the density Fourier sums rho(k)
(record_ftrho_unkorrigiert) against numpy FP64 on the same positions, and
against the reference's own observables (tests/golden/obs.npz)."""
import os

import numpy as np
import pytest

import configs as C
from conftest import GOLDEN, golden, gpos

pytestmark = pytest.mark.gpu
GOLDEN_OBS = os.path.join(GOLDEN, "obs.npz")


def _abs(p, pos):
    B = C.derived(p)["nachList_Breite"]
    return [pos[s][0] * B + pos[s][1] for s in (0, 1)]


@pytest.mark.parametrize("name", ["tiny_cic", "c1_cic"])
def test_pair_correlation_counts(gpu, name):
    p = C.CONFIGS[name]
    r = gpu.Run(p, seed=1)
    pos = gpos(golden(name), "init")
    r.set_positions(pos)
    x = _abs(p, r.get_positions())
    L, N1, N2 = p["L"], p["N1"], p["N2"]
    dr, bins = 0.2, int(0.5 * L / 0.2) + 1
    norm = {0: 2.0 / ((N1 - 1) * np.pi * (N1 / L / L) * dr * dr),
            1: 1.0 / ((N1 - 1) * np.pi * (N2 / L / L) * dr * dr),
            2: 2.0 / ((N2 - 1) * np.pi * (N2 / L / L) * dr * dr)}
    for which, (a, b, once) in enumerate([(0, 0, True), (0, 1, False), (1, 1, True)]):
        d = x[a][:, None, :] - x[b][None, :, :]
        d -= L * np.round(d / L)
        rr = np.sqrt((d ** 2).sum(-1))
        if once:
            rr = rr[np.tril_indices(len(x[a]), -1)]
        idx = (rr / dr).astype(int).ravel()
        want = np.bincount(idx[idx < bins], minlength=bins)
        g = r.korrelationsfunktion(which, dr, bins)
        got = np.rint(g * (2 * np.arange(bins) + 1) / norm[which]).astype(int)
        assert got.sum() == want.sum(), which
        assert np.abs(got - want).max() <= 2, which  # bin-edge rounding only
        assert np.abs(got - want).sum() <= 4, which


def test_density_fourier_sums(gpu):
    p = C.CONFIGS["c1_cic"]
    r = gpu.Run(p, seed=1)
    r.set_positions(gpos(golden("c1_cic"), "init"))
    x = _abs(p, r.get_positions())
    qbins, dq = 30, 4 * np.pi / p["L"]
    ii, jj = np.meshgrid(np.arange(qbins), np.arange(qbins), indexing="ij")
    disk = ii ** 2 + jj ** 2 <= qbins ** 2
    for s in (0, 1):
        want = np.exp(1j * dq * (x[s][:, 0, None, None] * ii + x[s][:, 1, None, None] * jj)).sum(0)
        want[~disk] = 0
        got = r.ftrho(s, qbins, dq)
        assert np.abs(got - want).max() <= 1e-9 * len(x[s])


def _qbin_sums(got, qbins, qabs2):
    """Per-(i, j) sums summed into the reference's |q|^2 bins (init_ftrho,
    auswertung.cpp:262-297: bins in order of first appearance)."""
    where = {int(q): k for k, q in enumerate(qabs2)}
    out = np.zeros(len(qabs2), complex)
    for i in range(qbins):
        for j in range(qbins):
            if i * i + j * j > qbins * qbins:
                break
            out[where[i * i + j * j]] += got[i, j]
    return out


@pytest.mark.parametrize("name", ["tiny_cic", "c1_cic"])
def test_observables_vs_reference(gpu, name):
    """g11/g12/g22 and rho(k) against the reference's own
    record_korrelationsfunktion11/12/22 and record_ftrho_unkorrigiert
    (tests/golden/obs.npz, made by the compiled reference). Pair counts
    equal up to pairs on a bin edge; rho(k) sums to 1e-9 N (FP64 sums in
    another order). Species-1 rho(k) on the set whose species-1 offsets are
    (r, r), where the reference's y-from-x-offset loop gives the true y."""
    g = dict(np.load(GOLDEN_OBS))
    p = C.CONFIGS[name]
    L, N1, N2 = p["L"], p["N1"], p["N2"]
    dr = 0.2
    for tag in ("a", "b"):
        pre = "%s_%s_" % (name, tag)
        pos = {s: (g[pre + "git%d" % s], g[pre + "rel%d" % s]) for s in (0, 1)}
        r = gpu.Run(p, seed=1)
        r.set_positions(pos)
        bins = len(g[pre + "g11"])
        norm = {0: 2.0 / ((N1 - 1) * np.pi * (N1 / L / L) * dr * dr),
                1: 1.0 / ((N1 - 1) * np.pi * (N2 / L / L) * dr * dr),
                2: 2.0 / ((N2 - 1) * np.pi * (N2 / L / L) * dr * dr)}
        for which, key in enumerate(("g11", "g12", "g22")):
            got = r.korrelationsfunktion(which, dr, bins)
            ref = g[pre + key]
            cg = np.rint(got * (2 * np.arange(bins) + 1) / norm[which]).astype(int)
            cr = np.rint(ref * (2 * np.arange(bins) + 1) / norm[which]).astype(int)
            print("%s %s %s: pairs %d, bins differing %d" % (name, tag, key, cr.sum(), (cg != cr).sum()))
            assert cg.sum() == cr.sum(), (tag, key)
            assert np.abs(cg - cr).max() <= 2 and np.abs(cg - cr).sum() <= 4, (tag, key)
            same = cg == cr
            assert np.allclose(got[same], ref[same], rtol=1e-12, atol=0), (tag, key)
        qbins, dq = 30, 4 * np.pi / L
        qabs2 = g[pre + "qabs2"]
        for s in ((1,) if tag == "a" else (0, 1)):
            got = _qbin_sums(r.ftrho(s, qbins, dq), qbins, qabs2)
            ref = g[pre + "ftrho%d_re" % (s + 1)] + 1j * g[pre + "ftrho%d_im" % (s + 1)]
            n = N1 if s == 0 else N2
            err = np.abs(got - ref).max()
            print("%s %s rho(k) species %d: max |diff| %.2e" % (name, tag, s + 1, err))
            assert err <= 1e-9 * n, (tag, s, err)
        r.close()
