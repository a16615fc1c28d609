"""bd_gridDensity_noalloc (the density deposit that allocates no device
memory) against the context entry points bd_gridDensity_* + bd_get_grid on
the same positions, through the C ABI. Both round every stencil term to the
same fixed-point integer and sum exactly, so the two densities are equal bit
for bit, which is what the test asserts. Two calls in a row share the
file-scope scratch array, so the second also shows that each call starts
from a cleared accumulator."""
import ctypes as ct

import numpy as np
import pytest

import configs as C
from conftest import golden, gpos, rel_l2


def _call(bd, params, scheme, dev, rho, nskipped, stream):
    ptr = lambda t: ct.c_void_p(t.data_ptr()) if t is not None else None
    return bd.lib().bd_gridDensity_noalloc(ct.byref(params), scheme, ptr(dev[0][0]), ptr(dev[0][1]),
                                           ptr(dev[1][0]), ptr(dev[1][1]), ptr(rho), ptr(nskipped),
                                           ct.c_void_p(stream))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny_ngp", "tiny_cic", "tiny_tsc", "c1_cic", "tiny_flags"])
def test_noalloc_deposit_matches_gridDensity(gpu, name):
    import torch
    p = C.CONFIGS[name]
    pos = gpos(golden(name), "init")
    params = gpu.params_from(p)
    run = gpu.Run(p, seed=1)
    run.set_positions(pos)
    Z = p["FFT_samples"]
    dev = {s: (torch.from_numpy(np.ascontiguousarray(pos[s][0], np.int32)).cuda() if p["N%d" % (s + 1)] else None,
               torch.from_numpy(np.ascontiguousarray(pos[s][1], np.float64)).cuda() if p["N%d" % (s + 1)] else None)
           for s in (0, 1)}
    rho = torch.empty(Z * Z, dtype=torch.float32, device="cuda")
    nskipped = torch.empty(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for scheme in (0, 1, 2):
        run.gridDensity(scheme)
        ref = run.grid(gpu.GRID_DENSITY).ravel()
        for rep in range(2):
            rho.fill_(float("nan"))
            nskipped.fill_(-1)
            st = _call(gpu, params, scheme, dev, rho, nskipped, stream)
            assert st == 0, gpu.BdError(st, "bd_gridDensity_noalloc")
            torch.cuda.synchronize()
            got = rho.double().cpu().numpy()
            assert int(nskipped.item()) == 0
            assert np.isfinite(got).all()
            err = rel_l2([got], [ref])
            print("%s scheme %d call %d: rel L2 %.2e, max |diff| %.2e" % (name, scheme, rep, err,
                                                                         np.abs(got - ref).max()))
            assert np.array_equal(got, ref)
    run.close()


@pytest.mark.gpu
def test_noalloc_one_species_null_pointers(gpu):
    """N2 == 0 with git2/rel2 and nskipped passed as NULL (documented as
    allowed), against bd_gridDensity_* of a one-species run."""
    import torch
    p = dict(C.CONFIGS["tiny_cic"], N2=0)
    pos = gpos(golden("tiny_cic"), "init")
    pos = {0: pos[0], 1: (np.zeros((0, 2), np.int32), np.zeros((0, 2)))}
    params = gpu.params_from(p)
    run = gpu.Run(p, seed=1)
    run.set_positions(pos)
    dev = {0: (torch.from_numpy(np.ascontiguousarray(pos[0][0], np.int32)).cuda(),
               torch.from_numpy(np.ascontiguousarray(pos[0][1], np.float64)).cuda()),
           1: (None, None)}
    Z = p["FFT_samples"]
    rho = torch.empty(Z * Z, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for scheme in (0, 1, 2):
        run.gridDensity(scheme)
        ref = run.grid(gpu.GRID_DENSITY).ravel()
        for rep in range(2):
            rho.fill_(float("nan"))
            st = _call(gpu, params, scheme, dev, rho, None, stream)
            assert st == 0, gpu.BdError(st, "bd_gridDensity_noalloc")
            torch.cuda.synchronize()
            assert np.array_equal(rho.double().cpu().numpy(), ref), (scheme, rep)
    run.close()


@pytest.mark.gpu
def test_noalloc_rejects_host_output(gpu):
    """rho must be device memory of the current device (the scratch array is
    per device): a host buffer is refused before any launch."""
    import torch
    p = C.CONFIGS["tiny_cic"]
    params = gpu.params_from(p)
    pos = gpos(golden("tiny_cic"), "init")
    dev = {s: (torch.from_numpy(np.ascontiguousarray(pos[s][0], np.int32)).cuda(),
               torch.from_numpy(np.ascontiguousarray(pos[s][1], np.float64)).cuda()) for s in (0, 1)}
    host_rho = torch.empty(p["FFT_samples"] ** 2, dtype=torch.float32)
    assert _call(gpu, params, 1, dev, host_rho, None, torch.cuda.current_stream().cuda_stream) == -1


@pytest.mark.gpu
def test_noalloc_counts_out_of_range_particles(gpu):
    import torch
    p = C.CONFIGS["tiny_cic"]
    pos = gpos(golden("tiny_cic"), "init")
    params = gpu.params_from(p)
    git = np.array(pos[0][0], np.int32)
    git[3] = (-1, 0)
    git[5] = (C.derived(p)["nachList_Zellen"], 2)
    dev = {0: (torch.from_numpy(git).cuda(), torch.from_numpy(np.array(pos[0][1])).cuda()),
           1: (torch.from_numpy(np.ascontiguousarray(pos[1][0], np.int32)).cuda(),
               torch.from_numpy(np.ascontiguousarray(pos[1][1], np.float64)).cuda())}
    Z = p["FFT_samples"]
    rho = torch.empty(Z * Z, dtype=torch.float32, device="cuda")
    nskipped = torch.empty(1, dtype=torch.int32, device="cuda")
    assert _call(gpu, params, 1, dev, rho, nskipped, torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    assert int(nskipped.item()) == 2


def test_noalloc_rejects_oversized_mesh(bdsim_mod):
    """A mesh larger than the scratch array is refused before any device work."""
    p = bdsim_mod.params_from(dict(C.CONFIGS["tiny_cic"], L=2200.0, FFT_samples=2048))
    st = bdsim_mod.lib().bd_gridDensity_noalloc(ct.byref(p), 1, ct.c_void_p(16), ct.c_void_p(16),
                                                ct.c_void_p(16), ct.c_void_p(16), ct.c_void_p(16),
                                                None, None)
    assert st == -3  # BD_ERR_UNSUPPORTED
    assert bdsim_mod.lib().bd_gridDensity_noalloc(ct.byref(p), 5, ct.c_void_p(16), ct.c_void_p(16),
                                                  None, None, ct.c_void_p(16), None, None) == -1
