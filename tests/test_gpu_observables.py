"""Observables computed on the device from the resident state: g11/g12/g22
(record_korrelationsfunktion*) and the density Fourier sums rho(k)
(record_ftrho_unkorrigiert) against numpy FP64 on the same positions."""
import numpy as np
import pytest

import configs as C
from conftest import golden, gpos

pytestmark = pytest.mark.gpu


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
