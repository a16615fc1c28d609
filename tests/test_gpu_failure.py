"""Failure detection on the device without a GPU fault: the fused step's
grid-barrier waits are bounded. A test hook makes one CTA leave instead of
arriving at a barrier and lowers the poll limit, so every other wait gives up
within microseconds; the kernel returns, the host reads BD_ERR_TIMEOUT at the
next synchronising call, and the run is back at its state before the step.
The reference has no such path (its routines print and return,
dynamik_methoden.cpp:80-83, 624-627, 1202)."""
import numpy as np
import pytest

import configs as C
from conftest import golden, gpos

pytestmark = pytest.mark.gpu

BD_ERR_TIMEOUT = -10


@pytest.mark.parametrize("barrier", [1, 2, 3])
def test_barrier_timeout_recovers_bit_identically(gpu, barrier):
    p = dict(C.CONFIGS["c1_cic"], noise_kind=gpu.NOISE_DISK)
    start = gpos(golden("c1_cic"), "start")
    a = gpu.Run(p, seed=99)
    b = gpu.Run(p, seed=99)
    for r in (a, b):
        r.set_positions(start)
        r.set_step(0)
        r.zeitschritte(7)
    assert a.launches_per_step() == 1  # the fused step
    a._call("bd_inject_barrier_timeout", barrier, 2000)
    with pytest.raises(gpu.BdError) as e:
        a.zeitschritte(1)
    assert e.value.status == BD_ERR_TIMEOUT
    # the failed step did not advance the run
    assert a.step_count() == 7 and a.time() == b.time()
    pa, pb = a.get_positions(), b.get_positions()
    for s in (0, 1):
        assert np.array_equal(pa[s][0], pb[s][0]) and np.array_equal(pa[s][1], pb[s][1])
    # the context is usable and steps on with the bits of the untouched run
    a.zeitschritte(40)
    b.zeitschritte(40)
    a.sync()
    pa, pb = a.get_positions(), b.get_positions()
    for s in (0, 1):
        assert np.array_equal(pa[s][0], pb[s][0]) and np.array_equal(pa[s][1], pb[s][1])
    assert a.step_count() == b.step_count() == 47 and a.time() == b.time()


def test_barrier_timeout_hook_arguments(gpu):
    p = dict(C.CONFIGS["c1_cic"])
    r = gpu.Run(p, seed=1)
    r.init_positions(1)
    for bad in ((0, 100), (4, 100), (1, 0)):
        with pytest.raises(gpu.BdError) as e:
            r._call("bd_inject_barrier_timeout", *bad)
        assert e.value.status == -1
    # a run the fused step does not cover (radix-3 mesh, adaptive dt)
    q = gpu.Run(C.CONFIGS["ref_default"], seed=1)
    q.init_positions(1)
    with pytest.raises(gpu.BdError) as e:
        q._call("bd_inject_barrier_timeout", 1, 100)
    assert e.value.status == -5
