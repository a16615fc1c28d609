"""TimestepInfo diagnostics (zeitschritt_debug's record of a step) and the
FP64 WCA energy and virial, against numpy FP64 on the same positions: the
pairs the reference's WCA loops examine (3x3 neighbour cells), the largest
force of each kind, the neighbour-list sizes of the largest-WCA particle, the
cell changes of the last step and the step length."""
import numpy as np
import pytest

import configs as C
from conftest import golden, gpos

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
