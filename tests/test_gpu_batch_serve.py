"""Batched stepping and the serving loop: a run's result is the same alone,
in a batch and in the served mix (bit for bit), admission respects the HBM
budget, cancellation and snapshots work, latency percentiles are reported."""
import numpy as np
import pytest

import configs as C
from conftest import golden, gpos

pytestmark = pytest.mark.gpu

MIX = ["tiny_cic", "tiny_tsc", "tiny_ngp", "c1_cic", "tiny_flags", "tiny_idgas"]


def _same(a, b):
    for s in (0, 1):
        assert np.array_equal(a[s][0], b[s][0])
        assert np.array_equal(a[s][1], b[s][1])


def test_batch_equals_single_runs(gpu):
    params = [dict(C.CONFIGS[n], noise_kind=gpu.NOISE_GAUSS) for n in MIX]
    seeds = [11 + k for k in range(len(MIX))]
    b = gpu.Batch(params, seeds)
    b.step(37)
    for k, (p, sd) in enumerate(zip(params, seeds)):
        r = gpu.Run(p, seed=sd)
        r.zeitschritte(37)
        _same(b.get_positions(k), r.get_positions())
        assert abs(b.time(k) - r.time()) <= 1e-12


@pytest.mark.parametrize("Z,scheme", [(256, 2), (512, 1), (1024, 0)])
def test_fused_step_equals_stage_kernels(gpu, Z, scheme):
    """The fused single-launch step gives the same positions, bit for bit, as
    the stage kernels (a fixed-dt run on a power-of-two mesh up to 1024^2)."""
    p = dict(C.CONFIGS["c1_cic"], N1=3000, N2=3000, L=180.0, FFT_samples=Z, densGrid_Schema=scheme,
             lambda_kapillar=20.0, noise_kind=gpu.NOISE_GAUSS)
    import oracle
    start = oracle.nonoverlap_positions(p, 5)
    a = gpu.Run(p, seed=21)
    b = gpu.Run(p, seed=21)
    a.set_positions(start)
    b.set_positions(start)
    assert a.launches_per_step() == 1  # the fused step
    a.zeitschritte(25)
    b.stage_times(25)  # the stage kernels, one step at a time
    _same(a.get_positions(), b.get_positions())
    assert a.time() == b.time()


def test_fused_step_after_outside_position_changes(gpu):
    """The fused step deposits the next step's density during its move; every
    other change of the positions (new positions, a debug step, a re-binning)
    must make the next fused step deposit afresh. The same sequence through
    the stage kernels gives the same bits."""
    p = dict(C.CONFIGS["c1_cic"], N1=2000, N2=2000, L=150.0, FFT_samples=256, densGrid_Schema=2,
             lambda_kapillar=20.0, noise_kind=gpu.NOISE_GAUSS)
    import oracle
    s1, s2 = oracle.nonoverlap_positions(p, 5), oracle.nonoverlap_positions(p, 6)
    a = gpu.Run(p, seed=21)
    b = gpu.Run(p, seed=21)
    assert a.launches_per_step() == 1
    for r, steps in ((a, a.zeitschritte), (b, b.stage_times)):
        r.set_positions(s1)
        steps(4)
        r.set_positions(s2)
        steps(3)
        r.zeitschritt_debug(0.02)
        steps(3)
        r.refresh_erwNachbar()
        steps(2)
    _same(a.get_positions(), b.get_positions())
    assert a.time() == b.time()


def test_batch_uneven_ensemble_runs(gpu):
    runs = C.batch_ensemble(12, seed=3)
    for q in runs:  # keep the test short
        q["N1"] = q["N2"] = min(q["N1"], 4000)
        q["noise_kind"] = gpu.NOISE_GAUSS
    b = gpu.Batch(runs, list(range(100, 112)))
    b.step(20)
    b.sync()
    for k in (0, 5, 11):
        pos = b.get_positions(k)
        for s in (0, 1):
            assert np.all(np.isfinite(pos[s][1]))


def _serve_until_done(srv, ids, max_ticks=10000):
    for _ in range(max_ticks):
        srv.tick()
        if all(srv.poll(i).state >= 2 for i in ids):
            return
    raise AssertionError("server did not finish")


def test_serving_result_same_alone_and_in_mix(gpu):
    target = dict(C.CONFIGS["c1_tsc"], noise_kind=gpu.NOISE_GAUSS)
    alone = gpu.Server(steps_per_tick=25)
    rid = alone.submit(target, seed=77, nsteps=130)
    _serve_until_done(alone, [rid])
    res_alone = alone.result(rid)
    mix = gpu.Server(steps_per_tick=25)
    others = []
    for k, n in enumerate(["tiny_cic", "tiny_ngp", "c1_cic"]):
        others.append(mix.submit(dict(C.CONFIGS[n], noise_kind=gpu.NOISE_GAUSS), seed=k, nsteps=60 + 40 * k))
    mix.tick()
    mix.tick()
    rid2 = mix.submit(target, seed=77, nsteps=130)  # arrives while others run
    others.append(mix.submit(dict(C.CONFIGS["tiny_tsc"], max_reisedistanz=1e30), seed=9, nsteps=90))
    _serve_until_done(mix, others + [rid2])
    _same(res_alone, mix.result(rid2))
    st = mix.stats()
    assert st.completed == 5 and st.p99_latency_s >= st.p50_latency_s > 0
    # the same run through the single-run API
    r = gpu.Run(target, seed=77)
    r.zeitschritte(130)
    _same(res_alone, r.get_positions())


def test_serving_positions_drawn_ahead(gpu):
    """Requests queued together have their initial positions drawn by the
    server's thread ahead of admission (a memory budget of three runs keeps
    the rest queued while the first ones step); each result equals the same
    run through the single-run API. A cancelled queued request is released
    while its positions may still be drawn."""
    p = dict(C.CONFIGS["c1_cic"], noise_kind=gpu.NOISE_GAUSS)
    one = gpu.footprint(gpu.params_from(p))
    srv = gpu.Server(hbm_budget=int(one * 3.5), steps_per_tick=20)
    ids = [srv.submit(p, seed=300 + k, nsteps=40 + 10 * (k % 3)) for k in range(9)]
    srv.cancel(ids[7])
    srv.release(ids[7])
    rest = [i for k, i in enumerate(ids) if k != 7]
    _serve_until_done(srv, rest)
    for k in (0, 4, 8):
        r = gpu.Run(p, seed=300 + k)
        r.zeitschritte(40 + 10 * (k % 3))
        _same(srv.result(ids[k]), r.get_positions())
        r.close()
    assert srv.stats().completed == 8


def test_serving_admission_budget_and_cancel(gpu):
    p = dict(C.CONFIGS["c1_cic"], noise_kind=gpu.NOISE_GAUSS)
    one = gpu.footprint(gpu.params_from(p))
    srv = gpu.Server(hbm_budget=int(one * 1.5), steps_per_tick=10)
    a = srv.submit(p, 1, 50)
    b = srv.submit(p, 2, 50)
    srv.tick()
    assert srv.poll(a).state == 1 and srv.poll(b).state == 0  # b waits for memory
    srv.cancel(a)
    assert srv.poll(a).state == 3
    srv.tick()
    assert srv.poll(b).state in (1, 2)
    _serve_until_done(srv, [b])
    assert srv.poll(b).state == 2
    big = dict(p, N1=10 ** 6, N2=10 ** 6, L=2000.0)
    with pytest.raises(gpu.BdError):
        srv.submit(big, 3, 10)


def test_serving_snapshots(gpu):
    p = dict(C.CONFIGS["tiny_cic"], noise_kind=gpu.NOISE_GAUSS)
    srv = gpu.Server(steps_per_tick=7)
    rid = srv.submit(p, 5, 45, snapshot_every=20)
    _serve_until_done(srv, [rid])
    st = srv.poll(rid)
    assert st.snapshots == 2 and st.steps_done == 45
    step, g, q = srv.snapshot(rid, 0)
    assert step == 40
    r = gpu.Run(p, seed=5)
    r.zeitschritte(40)
    ref = r.get_positions()
    assert np.array_equal(g, ref[0][0]) and np.array_equal(q, ref[0][1])


def test_serving_churn_reuses_memory(gpu):
    """Many runs joining and leaving: every request completes with the same
    bits as the single-run API, the budget accounting returns to zero, a
    second wave of the same requests needs no further device memory (the
    engine's pool reuses the arrays of retired runs), and the tick time split
    adds up."""
    import torch
    names = ["tiny_cic", "tiny_ngp", "tiny_tsc", "c1_cic"]
    reqs = [(dict(C.CONFIGS[names[k % 4]], noise_kind=gpu.NOISE_GAUSS, max_reisedistanz=1e30), 300 + k,
             5 + 7 * (k % 9)) for k in range(40)]  # serving steps with a fixed dt
    srv = gpu.Server(steps_per_tick=10)

    def wave():
        ids = []
        for k, (p, seed, n) in enumerate(reqs):
            ids.append(srv.submit(p, seed, n))
            if k % 5 == 4:
                srv.tick()
        _serve_until_done(srv, ids)
        return ids

    ids = wave()
    torch.cuda.synchronize()
    free_after_first = torch.cuda.mem_get_info()[0]
    for k in (0, 7, 13, 38):
        p, seed, n = reqs[k]
        r = gpu.Run(p, seed=seed)
        r.zeitschritte(n)
        _same(srv.result(ids[k]), r.get_positions())
        r.close()
    ids2 = wave()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] >= free_after_first - (64 << 20)
    st = srv.stats()
    assert st.completed == 2 * len(reqs) and st.active == 0 and st.hbm_in_use == 0
    assert st.particle_steps == 2 * sum((p["N1"] + p["N2"]) * n for p, _, n in reqs)
    assert st.step_s > 0 and st.host_s >= 0
    assert st.admit_s + st.plan_s + st.fetch_s <= st.host_s + 1e-3
    for i in ids + ids2:
        assert srv.poll(i).state == 2


def test_fused_phase_times(gpu):
    """bd_fused_phase_times: four positive phase times per step, from steps
    that are real steps (the same bits as the stage kernels); a run that does
    not use the fused step (mesh 48, radix 3) reports none."""
    import oracle
    p = dict(C.CONFIGS["c1_cic"], N1=3000, N2=3000, L=180.0, FFT_samples=256, densGrid_Schema=2,
             lambda_kapillar=20.0, noise_kind=gpu.NOISE_GAUSS)
    start = oracle.nonoverlap_positions(p, 5)
    a = gpu.Run(p, seed=3)
    a.set_positions(start)
    ph = a.fused_phase_times(5)
    assert list(ph) == gpu.FUSED_PHASES
    assert all(v > 0 for v in ph.values()) and sum(ph.values()) < 5.0  # ms per step
    b = gpu.Run(p, seed=3)
    b.set_positions(start)
    b.stage_times(5)
    _same(a.get_positions(), b.get_positions())
    q = gpu.Run(C.CONFIGS["tiny_cic"], seed=1)
    q.set_positions(gpos(golden("tiny_cic"), "init"))
    assert q.fused_phase_times(1) is None


@pytest.mark.parametrize("classic", [False, True])
def test_batch_autotune_keeps_bits(gpu, classic):
    """bd_batch_autotune times its candidate plans (transform items per
    launch for the pipelined step; deposit tiles x transform items for the
    classic stage kernels, here forced by a radix-3 mesh in the batch, with an
    adaptive-dt run), then the particle kernel's two shapes, keeps the fastest
    and changes no result: the tuned batch steps to the same bits as an
    untuned one (the timed particle launches leave no trace)."""
    runs = C.batch_ensemble(6, seed=5)
    for q in runs:  # keep the test short
        q["N1"] = q["N2"] = min(q["N1"], 3000)
        q["noise_kind"] = gpu.NOISE_GAUSS
    if classic:
        runs[2]["FFT_samples"] = 96
        runs[3]["max_reisedistanz"] = 0.05  # adaptive dt: forces and move in two launches
    seeds = list(range(40, 46))
    a = gpu.Batch(runs, seeds)
    b = gpu.Batch(runs, seeds)
    assert classic or a.launches_per_step() == 6
    a.step(5)
    b.step(5)
    res = a.autotune(3)
    print("autotune: tiles >= %d, items >= %d, largest tile %d, %d candidates, %.4f -> %.4f ms per mesh pass; "
          "particle kernel shape %d, %.4f -> %.4f ms"
          % (res.dep_tiles_min, res.fft_items_min, res.dep_tile_max, res.candidates, res.default_ms,
             res.best_ms, res.particle_shape, res.particle_default_ms, res.particle_best_ms))
    targets = (148, 296, 592, 1184, 2368, 4736)
    assert res.candidates == (16 if classic else 6) + 2  # plans, then the particle kernel's two shapes
    assert res.dep_tiles_min in targets and res.fft_items_min in targets and res.dep_tile_max >= 16
    assert res.default_ms > 0 and 0 < res.best_ms <= res.default_ms
    assert res.particle_shape in (0, 1) and 0 < res.particle_best_ms <= res.particle_default_ms
    a.step(20)
    b.step(20)
    for k in range(len(runs)):
        _same(a.get_positions(k), b.get_positions(k))


# runs on power-of-two meshes with a fixed dt: the pipelined stage step
PIPE_MIX = ["tiny_ngp", "c1_cic", "tiny_flags", "tiny_radial", "c1_ngp", "c1_tsc"]


# the pipelined step's forms: six launches on two streams, or the particle
# kernel and one cooperative launch (at 2, 3 or 4 CTAs per SM)
FORMS = [(0, 0, 6), (1, 2, 2), (1, 3, 2), (1, 4, 2)]


@pytest.mark.parametrize("form,ctas,launches", FORMS)
def test_pipelined_batch_equals_single_runs(gpu, form, ctas, launches):
    """A batch of runs on power-of-two meshes steps with the pipelined stage
    step (the density deposited in the move, the next transform beside the
    cell sort), in either form; every run ends with the bits of the same run
    stepped alone (the fused step), through the 16-step graph and single
    steps."""
    params = [dict(C.CONFIGS[n], noise_kind=gpu.NOISE_GAUSS) for n in PIPE_MIX]
    seeds = [31 + k for k in range(len(PIPE_MIX))]
    b = gpu.Batch(params, seeds)
    b.set_step_form(form, ctas)
    assert b.launches_per_step() == launches
    b.step(37)
    for k, (p, sd) in enumerate(zip(params, seeds)):
        r = gpu.Run(p, seed=sd)
        assert r.launches_per_step() == 1
        r.zeitschritte(37)
        _same(b.get_positions(k), r.get_positions())
        assert b.time(k) == r.time()


@pytest.mark.parametrize("form", [0, 1])
def test_pipelined_step_equals_stage_kernels(gpu, form):
    """The pipelined stage step against the classic stage kernels (deposit
    tiles, one transform launch per pass and mesh size, separate chunk scan)
    on a batch with meshes up to 2048^2 (six launches: the two-launch form
    takes meshes up to 1024^2), the same bits after steps, position changes
    and more steps; then an ensemble in the chosen form."""
    import oracle
    p = dict(C.CONFIGS["c1_cic"], N1=3000, N2=3000, L=180.0, FFT_samples=2048, densGrid_Schema=2,
             lambda_kapillar=20.0, noise_kind=gpu.NOISE_GAUSS)
    q = dict(p, FFT_samples=128, densGrid_Schema=1)
    s1, s2 = oracle.nonoverlap_positions(p, 5), oracle.nonoverlap_positions(p, 6)
    a = gpu.Batch([p, q], [21, 22])
    b = gpu.Batch([p, q], [21, 22])
    a.set_step_form(form)
    assert a.launches_per_step() == 6
    for r, steps in ((a, a.step), (b, b.stage_times)):
        for k in (0, 1):
            r.set_positions(k, s1)
        steps(19)
        r.set_positions(0, s2)
        steps(6)
    for k in (0, 1):
        _same(a.get_positions(k), b.get_positions(k))
        assert a.time(k) == b.time(k)
    runs = C.batch_ensemble(5, seed=9)
    for q in runs:
        q["N1"] = q["N2"] = min(q["N1"], 3000)
        q["noise_kind"] = gpu.NOISE_DISK
    seeds = list(range(60, 65))
    A = gpu.Batch(runs, seeds)
    B = gpu.Batch(runs, seeds)
    A.set_step_form(form)
    assert A.launches_per_step() == (2 if form else 6)
    A.step(23)
    B.stage_times(23)
    for k in range(len(runs)):
        _same(A.get_positions(k), B.get_positions(k))
        assert A.time(k) == B.time(k)


def test_pipelined_serving_uneven_budgets(gpu):
    """A served mix on the pipelined stage step whose runs have different
    step budgets (runs wait at their budget while others step, join while
    others run, and leave): every result has the bits of the single-run API."""
    names = ["c1_cic", "tiny_ngp", "c1_ngp", "c1_tsc", "tiny_flags"]
    reqs = [(dict(C.CONFIGS[names[k % 5]], noise_kind=gpu.NOISE_DISK), 500 + k, 3 + 11 * (k % 7))
            for k in range(15)]
    srv = gpu.Server(steps_per_tick=10)
    ids = []
    for k, (p, seed, n) in enumerate(reqs):
        ids.append(srv.submit(p, seed, n, snapshot_every=20))
        if k % 4 == 3:
            srv.tick()
    _serve_until_done(srv, ids)
    for k in range(len(reqs)):
        p, seed, n = reqs[k]
        r = gpu.Run(p, seed=seed)
        r.zeitschritte(n)
        _same(srv.result(ids[k]), r.get_positions())
        r.close()


def test_serving_autotunes_large_mix(gpu):
    """Once the resident mix holds 2^20 particles the server runs the batch
    autotuner on it (counted in plan_s); results are those of the same runs
    through the single-run API, bit for bit."""
    import math
    reqs = []
    for k, n in enumerate((300000, 280000)):
        L = math.sqrt(2 * n * math.pi / (4 * 0.2))
        z = 2 ** int(round(math.log2(L / 2)))
        reqs.append((dict(C.CONFIGS["c1_tsc"], N1=n, N2=n, L=L, FFT_samples=z, lambda_kapillar=L / 8,
                          noise_kind=gpu.NOISE_GAUSS, max_reisedistanz=1e30), 500 + k, 12 + 5 * k))
    srv = gpu.Server(steps_per_tick=8)
    ids = [srv.submit(p, sd, n) for p, sd, n in reqs]
    _serve_until_done(srv, ids)
    assert srv.stats().plan_s > 0
    for (p, sd, n), rid in zip(reqs, ids):
        r = gpu.Run(p, seed=sd)
        r.zeitschritte(n)
        _same(srv.result(rid), r.get_positions())
        r.close()


def test_batch_positions_both_species_at_once(gpu):
    """bd_batch_set_positions_all / bd_batch_get_positions_all (one copy and
    one sort for both species of a run) against the per-species calls: the
    same positions read back, and the same bits after further steps."""
    params = [dict(C.CONFIGS[n], noise_kind=gpu.NOISE_GAUSS) for n in ("tiny_cic", "c1_tsc", "tiny_ngp")]
    seeds = [61, 62, 63]
    src = gpu.Batch(params, seeds)
    src.step(10)
    pos = src.get_positions(1)
    for s in (0, 1):
        g, r = src.get_positions_species(1, s)
        assert np.array_equal(g, pos[s][0]) and np.array_equal(r, pos[s][1])
    a = gpu.Batch(params, seeds)
    b = gpu.Batch(params, seeds)
    a.set_positions(1, pos)
    for s in (0, 1):
        b.set_positions_species(1, s, pos[s][0], pos[s][1])
    _same(a.get_positions(1), pos)
    a.step(15)
    b.step(15)
    for k in range(3):
        _same(a.get_positions(k), b.get_positions(k))
