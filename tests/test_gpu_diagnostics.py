"""TimestepInfo diagnostics (zeitschritt_debug's record of a step) and the
FP64 WCA energy and virial, against numpy FP64 on the same positions: the
pairs the reference's WCA loops examine (3x3 neighbour cells), the largest
force of each kind, the neighbour-list sizes of the largest-WCA particle, the
cell changes of the last step and the step length."""
import numpy as np
import pytest

import configs as C
from conftest import abs_pos, golden, gpos, min_image

pytestmark = pytest.mark.gpu


def _reference(p, pos):
    d = C.derived(p)
    Cn, B = d["nachList_Zellen"], d["nachList_Breite"]
    sp = np.concatenate([np.zeros(p["N1"], int), np.ones(p["N2"], int)])
    git = np.concatenate([pos[0][0], pos[1][0]]).astype(int)
    rel = np.concatenate([pos[0][1], pos[1][1]])
    # cell step from i to j, wrapped to -1, 0, 1 (others are not neighbours)
    dc = (git[None, :, :] - git[:, None, :] + Cn) % Cn
    dc = np.where(dc == Cn - 1, -1, dc)
    near = (np.abs(dc) <= 1).all(-1)
    np.fill_diagonal(near, False)
    same = sp[:, None] == sp[None, :]
    examined = (near & (same | (sp[:, None] == 0))).sum()
    dxy = (rel[:, None, :] - rel[None, :, :]) - dc * B
    t = np.where(same, sp[:, None], 2)
    sig = np.array([1.0, p["sigma11_22"], p["sigma11_12"]])[t]
    eps = np.array([1.0, p["eps22_11"], p["eps12_11"]])[t]
    a2s = (dxy ** 2).sum(-1) * sig ** 2
    inside = near & (a2s <= 2 ** (1 / 3))
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        i6 = 1.0 / a2s ** 3
        U = 4 * eps * (i6 * i6 - i6) + eps
        f = np.minimum(24 * eps * sig * i6 / a2s * (2 * i6 - 1), p["maxPairWCA"])
        W = f * a2s / sig
    return examined, 0.5 * U[inside].sum(), 0.5 * W[inside].sum(), git, sp, Cn


@pytest.mark.parametrize("name", ["tiny_cic", "c1_cic", "tiny_tsc"])
def test_timestep_info(gpu, name):
    p = dict(C.CONFIGS[name], noise_kind=gpu.NOISE_GAUSS)
    r = gpu.Run(p, seed=3)
    r.set_positions(gpos(golden(name), "init"))
    before = r.get_positions()
    r.zeitschritt()
    after = r.get_positions()
    info = r.timestep_info()
    # forces of the current positions, as the info call computed them
    f = r.get_forces()
    examined, E, W, git, sp, Cn = _reference(p, after)
    assert info["num_WCA_berechnet"] == examined
    # FP64 sums; the pair prefactors are the FP32 ones of the force kernels
    assert info["E_WCA"] == pytest.approx(E, rel=1e-6, abs=1e-9)
    assert info["virial_WCA"] == pytest.approx(W, rel=1e-6, abs=1e-9)
    for kind, key in (("wca", "WCA"), ("kap", "Kap"), ("noise", "RND")):
        a = np.concatenate([f[(kind, 0)], f[(kind, 1)]])
        m2 = (a ** 2).sum(1)
        k = info["max%sindex" % key] + (0 if info["max%stype" % key] == 1 else p["N1"])
        # the reported particle carries the largest force (ties and FP32 rounding aside)
        assert m2[k] >= m2.max() * (1 - 1e-6), key
        assert (info["max%sx" % key], info["max%sy" % key]) == (a[k, 0], a[k, 1])
    # neighbour-list sizes of the largest-WCA particle
    k = info["maxWCAindex"] + (0 if info["maxWCAtype"] == 1 else p["N1"])
    dc = (git - git[k] + Cn) % Cn
    nb = ((dc <= 1) | (dc == Cn - 1)).all(1)
    assert (info["maxWCA_numWW1"], info["maxWCA_numWW2"]) == (int((nb & (sp == 0)).sum()),
                                                              int((nb & (sp == 1)).sum()))
    # cell changes of the step just taken
    for s in (0, 1):
        moved = int((before[s][0] != after[s][0]).any(1).sum())
        assert info["num_Zellwechsel%d" % (s + 1)] == moved
    if p["max_reisedistanz"] >= 1e20:
        assert info["dt"] == p["dt_max"]
    else:
        assert info["dt"] == pytest.approx(r.optimaler_zeitschritt(), rel=1e-7)


@pytest.mark.parametrize("name", ["tiny_cic", "tiny_tsc"])
def test_zeitschritt_debug_vs_oracle(gpu, oracle_mod, name):
    """zeitschritt_debug(mrd): the step length optimaler_zeitschritt(mrd)
    (also for a fixed-dt run), the move, and its TimestepInfo, against the
    oracle's step with the same travel bound and the same Philox disk noise,
    over travel bounds from above the run's own to far below."""
    p = dict(C.CONFIGS[name], noise_kind=gpu.NOISE_DISK)
    start = gpos(golden(name), "start")
    B, L = C.derived(p)["nachList_Breite"], p["L"]
    r = gpu.Run(p, seed=99)
    r.set_positions(start)
    r.set_step(0)
    o = oracle_mod.Oracle(p, 1)
    o.set_positions(start)
    o.set_noise(oracle_mod.NOISE_PHILOX_DISK, 99)
    o.set_step(0)
    for mrd in (0.5, 0.05, 0.01, 0.003):
        for _ in range(5):
            before = r.get_positions()
            info = r.zeitschritt_debug(mrd)
            after = r.get_positions()
            dto = o.step_mrd(mrd)
            assert info["dt"] == pytest.approx(dto, rel=1e-4), (mrd, info["dt"], dto)
            assert info["dt"] <= p["dt_max"] * (1 + 1e-7)  # stored in FP32
            of = o.get_forces()  # the forces of the step just taken
            w = np.concatenate([of[("wca", 0)], of[("wca", 1)]])
            m2 = (w ** 2).sum(1)
            k = info["maxWCAindex"] + (0 if info["maxWCAtype"] == 1 else p["N1"])
            assert m2[k] >= m2.max() * (1 - 1e-4)
            assert np.hypot(info["maxWCAx"], info["maxWCAy"]) == pytest.approx(np.sqrt(m2.max()), rel=1e-4)
            for s in (0, 1):
                moved = int((before[s][0] != after[s][0]).any(1).sum())
                assert info["num_Zellwechsel%d" % (s + 1)] == moved
        a = abs_pos(r.get_positions(), B)
        b = abs_pos(o.get_positions(), B)
        dd = np.concatenate([min_image(a[s] - b[s], L) for s in (0, 1)])
        print("%s mrd %g: dt %.3e, position rms %.2e max %.2e" % (name, mrd, info["dt"],
                                                                   np.sqrt((dd ** 2).mean()), np.abs(dd).max()))
        assert np.sqrt((dd ** 2).mean()) <= 1e-3 and np.abs(dd).max() <= 2e-2
    r.close()


def test_bdkap_debugmode_sweep(gpu, tmp_path):
    """The driver's debugmode travel-distance sweep (main.cpp:156-218):
    mrd_data1.txt / mrd_data2.txt with the reference's header lines and one
    line per mrd = 0.95^k > 0.01; the largest WCA force is recorded (the
    reference's debug routines leave it at zero) and the mean step shrinks
    with the travel bound."""
    import os
    import subprocess
    import build_ref
    from scipy.stats import spearmanr
    exe = os.path.join(os.path.dirname(gpu.LIB_PATH), "bdkap")
    p = dict(C.CONFIGS["tiny_cic"], N1=150, N2=100, L=28.0, FFT_samples=32)
    text = build_ref.parameter_h(p).replace("const bool debugmode = false;", "const bool debugmode = true;")
    (tmp_path / "parameter.h").write_text(text)
    res = subprocess.run([exe, str(tmp_path / "parameter.h"), "--seed", "5", "--out", str(tmp_path)],
                         cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    mrd = [1.0]
    while mrd[-1] * 0.95 > 0.01:
        mrd.append(mrd[-1] * 0.95)
    for f, head in (("mrd_data1.txt", "# Mittelwerte über 50 Zeitschritte. Früh = erste 50 Zeitschritte. "),
                    ("mrd_data2.txt", "# Mittelwerte über 50 Zeitschritte. Spät = nach 1000 Zeitschritten ")):
        lines = (tmp_path / f).read_text().split("\n")
        assert lines[0] == head
        assert lines[1] == "# Format: mrd TAB <F_WCA_max> TAB |F_WCA_highest| TAB dt " and lines[2] == ""
        rows = np.array([[float(v) for v in l.split(" \t ")] for l in lines[3:] if l.strip()])
        assert rows.shape == (len(mrd), 4)
        np.testing.assert_allclose(rows[:, 0], mrd, rtol=1e-5)
        assert (rows[:, 1] > 0).all() and (rows[:, 2] >= rows[:, 1] * (1 - 1e-5)).all()
        assert (rows[:, 3] <= p["dt_max"] * (1 + 1e-6)).all() and rows[-1, 3] < 0.05 * rows[0, 3]
        # every mrd starts from a fresh random start, so the means are noisy
        # (overlaps set the force bound) and the large bounds all give dt_max;
        # the step still falls with the travel bound
        rho = spearmanr(rows[:, 0], rows[:, 3]).correlation
        print(f, "rank correlation of dt with mrd %.3f" % rho)
        assert rho >= 0.7
        assert rows[-10:, 3].mean() < 0.05 * rows[:10, 3].mean()
