"""The oracle (C restatement, oracle/bd_oracle.c) pinned against the
reference's own outputs (tests/golden, produced by the compiled reference),
against known-answer vectors and against numpy. CPU only."""
import numpy as np
import pytest

import configs as C
from conftest import K1_TOL, golden, gpos, k1_pair_case, pair_forces

GOLDEN_CONFIGS = ["tiny_ngp", "tiny_cic", "tiny_tsc", "tiny_radial", "tiny_flags", "tiny_idgas",
                  "ref_default", "c1_cic", "c1_ngp", "c1_tsc"]


@pytest.mark.parametrize("name", GOLDEN_CONFIGS)
def test_init_positions_bit_exact(oracle_mod, name):
    """init_zufallspos with the reference's mt19937_64 stream, incl. the
    (int) x / B cell rounding (dynamik_methoden.cpp:1655-1656)."""
    g = golden(name)
    o = oracle_mod.Oracle(C.CONFIGS[name], 7)
    o.init_positions(C.CONFIGS[name]["startpos_methode"])
    pos = o.get_positions()
    ref = gpos(g, "init")
    for s in (0, 1):
        assert np.array_equal(pos[s][0], ref[s][0])
        assert np.array_equal(pos[s][1], ref[s][1])


@pytest.mark.parametrize("name", GOLDEN_CONFIGS)
def test_forces_bit_exact(oracle_mod, name):
    g = golden(name)
    p = C.CONFIGS[name]
    o = oracle_mod.Oracle(p, 1)
    o.set_positions(gpos(g, "init"))
    f = o.forces()
    for kind in ("wca", "kap"):
        for s in (0, 1):
            assert np.array_equal(f[(kind, s)], g["forces_%s%d" % (kind, s)]), (kind, s)
    if "grid_rho" in g and not p["idgas_only"]:  # idgas_only never fills the grids
        assert np.array_equal(o.grid(0), g["grid_rho"])
        assert np.array_equal(o.grid(1), g["grid_Fx"])
        assert np.array_equal(o.grid(2), g["grid_Fy"])
    assert o.oob() == 0


@pytest.mark.parametrize("name", GOLDEN_CONFIGS)
def test_injected_noise_trajectory_bit_exact(oracle_mod, name):
    """zeitschritt with identical injected noise: the oracle reproduces the
    reference trajectory bit for bit, including re-binning."""
    g = golden(name)
    p = C.CONFIGS[name]
    o = oracle_mod.Oracle(p, 1)
    o.set_positions(gpos(g, "start"))
    o.set_noise(oracle_mod.NOISE_PHILOX_DISK, 99)
    o.set_step(0)
    every = int(g["traj_every"])
    k = 0
    t = 0.0
    while "traj%d_git0" % k in g:
        t += o.step(every)
        q = o.get_positions()
        ref = gpos(g, "traj%d" % k)
        for s in (0, 1):
            assert np.array_equal(q[s][0], ref[s][0]), (k, s)
            assert np.array_equal(q[s][1], ref[s][1]), (k, s)
        # the checker sums dt step by step, this loop per chunk
        assert abs(t - float(g["traj%d_t" % k])) <= 1e-12 * abs(t)
        k += 1
    assert k >= 1


def test_noiseless_trajectory_bit_exact(oracle_mod):
    g = golden("c1_cic")
    o = oracle_mod.Oracle(C.CONFIGS["c1_cic"], 1)
    o.set_positions(gpos(g, "start"))
    o.set_noise(oracle_mod.NOISE_NONE)
    every = int(g["traj_every"])
    k = 0
    while "noiseless%d_git0" % k in g:
        o.step(every)
        q = o.get_positions()
        ref = gpos(g, "noiseless%d" % k)
        for s in (0, 1):
            assert np.array_equal(q[s][1], ref[s][1])
        k += 1
    assert k == 4


def test_neighbour_lists_match_reference(oracle_mod):
    """erwNachbarn after WCA_init (dynamik_methoden.cpp:459-526)."""
    g = golden("tiny_cic")
    p = C.CONFIGS["tiny_cic"]
    o = oracle_mod.Oracle(p, 1)
    o.set_positions(gpos(g, "init"))
    Cn = C.derived(p)["nachList_Zellen"]
    for s in (0, 1):
        lens = g["lists_len%d" % s]
        ids = g["lists_ids%d" % s]
        off = 0
        for i in range(Cn):
            for j in range(Cn):
                n = lens[i * Cn + j]
                assert np.array_equal(o.list(s, i, j), ids[off:off + n])
                off += n


def test_fft_shim_matches_numpy(oracle_mod):
    """The FFTW-API shim (sign conventions, mixed radix incl. 3) vs numpy."""
    rng = np.random.default_rng(0)
    for Z in (8, 12, 48, 64, 96):
        p = dict(C.CONFIGS["tiny_cic"], FFT_samples=Z)
        o = oracle_mod.Oracle(p, 1)
        o.set_positions({0: (np.zeros((p["N1"], 2), np.int32), rng.uniform(0, 1, (p["N1"], 2))),
                         1: (np.zeros((p["N2"], 2), np.int32), rng.uniform(0, 1, (p["N2"], 2)))})
        o.forces()
        rho = o.grid(0)
        # reference pipeline with numpy: F = ifft2(i*sinG*fft2(rho))
        d = C.derived(p)
        dx, dq = d["densGrid_Breite"], d["dq"]
        q = dq * (((np.arange(Z) + Z // 2) % Z) - 0.5 * Z)
        qx, qy = np.meshgrid(q, q, indexing="ij")
        lam = p["lambda_kapillar"]
        G = 1.0 / (4 * np.sin(0.5 * qx * dx) ** 2 / dx / dx + 4 * np.sin(0.5 * qy * dx) ** 2 / dx / dx + 1.0 / lam ** 2)
        if lam > 0.2 * p["L"]:
            G[0, 0] = 0.0
        sx = p["kapillar_vorfaktor"] * np.sin(qx * dx) / dx * G / Z / Z
        rk = np.fft.fft2(rho)
        Fx = np.fft.ifft2(1j * sx * rk) * Z * Z
        assert np.max(np.abs(Fx.real - o.grid(1))) < 1e-12 * max(1.0, np.max(np.abs(Fx.real)))


def test_philox_known_answers(oracle_mod):
    """Philox4x32-10 known-answer vectors (Salmon et al., SC11)."""
    import ctypes as ct
    L = oracle_mod.lib()
    cases = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in cases:
        c = (ct.c_uint32 * 4)(*ctr)
        k = (ct.c_uint32 * 2)(*key)
        out = (ct.c_uint32 * 4)()
        L.bdo_philox4x32_10(c, k, out)
        assert tuple(out) == want


def test_philox_noise_distributions(oracle_mod):
    xi = oracle_mod.philox_noise(5, 0, 20000, 20000, gauss=False)
    r2 = (xi ** 2).sum(1)
    assert r2.max() <= 5.0 + 1e-12
    assert abs(xi.var(0).mean() - 1.25) < 0.02  # uniform disk of radius sqrt 5
    g = oracle_mod.philox_noise(5, 0, 20000, 20000, gauss=True)
    assert abs(g.mean()) < 0.02 and abs(g.var() - 1.0) < 0.02


LOCALDENS_CONFIGS = ["tiny_cic", "tiny_tsc", "tiny_radial", "c1_cic"]


@pytest.mark.parametrize("name", LOCALDENS_CONFIGS)
def test_local_density_matches_reference_analysis(oracle_mod, name):
    """Local-density grids, histograms and threshold counts
    (main_auswertung.cpp:182-390) against the reference's own analysis
    program (tests/golden/localdens.npz): counts bit-exact, grids to the
    %g precision the program prints them with (relative 5e-6)."""
    z = golden("localdens")
    L = C.CONFIGS[name]["L"]
    for f in (0, 1):
        key = "%s_f%d_" % (name, f)
        x1 = z[key + "x1"].astype(np.float64)
        x2 = z[key + "x2"].astype(np.float64)
        g1, g2 = oracle_mod.lokale_dichte(L, x1, x2)
        n = oracle_mod.snapgrid_num(L)
        assert g1.shape == (n, n)
        w = L / n
        assert abs(g1.sum() * w * w - len(x1)) < 1e-9 * len(x1)
        assert abs(g2.sum() * w * w - len(x2)) < 1e-9 * max(len(x2), 1)
        if key + "g1" in z:
            for g, ref in ((g1, z[key + "g1"]), (g2, z[key + "g2"])):
                ref = ref.astype(np.float64)
                assert np.all(np.abs(g - ref) <= 5.01e-6 * np.abs(g) + 1e-30)
        hist, over = oracle_mod.rhohist(g1, g2)
        assert np.array_equal(hist, z[key + "hist"])
        assert np.array_equal(over, z[key + "over"])
        assert (hist.sum(1) == n * n).all()


@pytest.mark.parametrize("scheme", [0, 1, 2])
def test_pair_capillary_force_k1_law(oracle_mod, scheme):
    """krafttestmode's known answer (main.cpp:220-248): an isolated pair
    attracts with gamma/(2π)·K1(r/lam)/lam along the line joining it,
    equal and opposite on the two particles."""
    for r in (3.0, 5.0, 8.0, 12.0, 20.0):
        for ang in (0.0, 0.7):
            p, pos, expect = k1_pair_case("c1_cic", scheme, r, ang)
            o = oracle_mod.Oracle(p, 1)
            o.set_positions(pos)
            f0, f1 = pair_forces(o.forces(), (0, 0))
            err = np.linalg.norm(f1 - expect) / np.linalg.norm(expect)
            assert err < K1_TOL[scheme], (r, ang, err)
            assert np.linalg.norm(f0 + f1) < 1e-9 * np.linalg.norm(expect)


@pytest.mark.parametrize("f2", [0.6, 2.5])
def test_pair_capillary_force_species_weights(oracle_mod, f2):
    """Species-2 particles deposit and feel the field with weight f2_f1
    (gridRoutinen.cpp:73, 122-123), so a 1-2 pair attracts with f2_f1 times
    the 1-1 force. (A 2-2 pair alone would need N1 = 0, which parameter.h:13
    rules out.)"""
    for r in (4.0, 9.0):
        p, pos, expect = k1_pair_case("c1_cic", 2, r, 0.4, species=(0, 1), f2=f2)
        o = oracle_mod.Oracle(p, 1)
        o.set_positions(pos)
        f0, f1 = pair_forces(o.forces(), (0, 1))
        assert np.linalg.norm(f1 - expect) / np.linalg.norm(expect) < K1_TOL[2]
        assert np.linalg.norm(f0 + f1) < 1e-9 * np.linalg.norm(expect)


@pytest.mark.parametrize("name", ["tiny_cic", "c1_cic"])
def test_observables_fixture_restated(name):
    """The reference's g11/g12/g22 and binned rho(k) (tests/golden/obs.npz,
    record_korrelationsfunktion11/12/22 and record_ftrho_unkorrigiert,
    auswertung.cpp:110-188, 262-375) restated in numpy: pair counts per bin
    of (int)(r / korr_dr), each pair once (12: all type-1 x type-2 pairs),
    weighted vorfaktor / (2b + 1); rho(k) summed over the (i, j) of one
    |q|^2. Species 1's rho(k) takes y from the x offset (auswertung.cpp:333)."""
    import os
    from conftest import GOLDEN
    g = dict(np.load(os.path.join(GOLDEN, "obs.npz")))
    p = C.CONFIGS[name]
    L, N1, N2 = p["L"], p["N1"], p["N2"]
    B = C.derived(p)["nachList_Breite"]
    dr = 0.2
    for tag in ("a", "b"):
        pre = "%s_%s_" % (name, tag)
        git = [g[pre + "git%d" % s] for s in (0, 1)]
        rel = [g[pre + "rel%d" % s] for s in (0, 1)]
        x = [git[s] * B + rel[s] for s in (0, 1)]
        bins = len(g[pre + "g11"])
        rho = (N1 / L / L, N2 / L / L)
        vor = {"g11": 2.0 / ((N1 - 1) * np.pi * rho[0] * dr * dr),
               "g12": 1.0 / ((N1 - 1) * np.pi * rho[1] * dr * dr),
               "g22": 2.0 / ((N2 - 1) * np.pi * rho[1] * dr * dr)}
        for key, (a, b, once) in (("g11", (0, 0, True)), ("g12", (0, 1, False)), ("g22", (1, 1, True))):
            d = x[a][:, None, :] - x[b][None, :, :]
            d -= L * np.round(d / L)
            rr = np.sqrt((d ** 2).sum(-1))
            if once:
                rr = rr[np.tril_indices(len(x[a]), -1)]
            idx = (rr / dr).astype(int).ravel()
            want = np.bincount(idx[idx < bins], minlength=bins)
            got = np.rint(g[pre + key] * (2 * np.arange(bins) + 1) / vor[key]).astype(int)
            assert np.abs(got - want).sum() <= 4, (tag, key)
        qbins, dq = 30, 4 * np.pi / L
        qabs2 = g[pre + "qabs2"]
        where = {int(q): k for k, q in enumerate(qabs2)}
        ys = [git[0][:, 1] * B + rel[0][:, 0], x[1][:, 1]]
        for s in (0, 1):
            want = np.zeros(len(qabs2), complex)
            for i in range(qbins):
                for j in range(qbins):
                    if i * i + j * j > qbins * qbins:
                        break
                    want[where[i * i + j * j]] += np.exp(1j * dq * (x[s][:, 0] * i + ys[s] * j)).sum()
            ref = g[pre + "ftrho%d_re" % (s + 1)] + 1j * g[pre + "ftrho%d_im" % (s + 1)]
            assert np.abs(want - ref).max() <= 1e-9 * len(x[s]), (tag, s)
