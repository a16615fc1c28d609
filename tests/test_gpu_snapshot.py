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
