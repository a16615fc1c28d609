#!/usr/bin/env python
"""Benchmark of the B200 Brownian-dynamics timestep (libbd_b200.so).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload medium|large|served]

Workload (`value`, `e2e`, `roofline`): the single-run medium configuration:
2D periodic box L=512, N1=N2=32768, TSC on a 512^2 mesh, lambda=64, Gamma=1
(kapillar_vorfaktor = 2 pi), q2 = 0.5, D = 1, dt = 5e-5, the reference's
uniform-disk noise (both arms draw the same distribution); positions
uniform-random from a seed with pairs closer than 0.8 sigma re-drawn (both
arms start from the same positions: from overlapping starts the reference's
fixed-dt update moves particles by several cells per step and then writes
outside its density array). Metric: particle-steps/s.
  value : device-resident steps, CUDA events on the library's stream, the L2
          flushed (256 MB write) before every timed step; summed event time
  e2e   : the reference-facing C ABI with host buffers: bd_set_positions_all
          (host -> device), K x bd_zeitschritt (one call per step, dt back to
          the host), bd_get_positions_all (device -> host); wall clock,
          the median of five repetitions of the sequence
Extras in the same line, each at its stated size and step count: the plain
small run (L=100, N=2000, CIC 128^2, 1000 steps), the batched ensemble of 256
uneven runs (5000 steps), the large single run (L=2896, N=2^21, TSC 2048^2,
2000 steps), and a served Poisson stream below the server's capacity (the
serving workload's request sizes and step counts, arrivals slow enough that
p50/p99 measure service, not queueing).
--workload served prints the served stream as the serving workload states
it (Poisson 50/s for 60 s, N1=N2 log-uniform in [1024, 262144], steps
log-uniform in [1e3, 1e5], snapshots every 1000 steps) with p50/p99.
With --gpus N (torchrun), every rank runs its own replica (the single-run
path does not shard) and its own share of the ensemble runs; times are the
max over ranks.
--impl reference times the reference's own CPU code (the compiled reference
under oracle/_ref, else the oracle port) with one process per host core, with
the same steps and warm-up as the GPU arm.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "bd-simulations_b200"))

METRIC = "particle-steps/s, batched+served vs plain, 1 B200 @ rel force err<=1e-5; p99"
TWO_PI = 2.0 * math.pi

C2 = dict(N1=32768, N2=32768, L=512.0, densGrid_Schema=2, FFT_samples=512, lambda_kapillar=64.0,
          kapillar_vorfaktor=TWO_PI, T=1.0, dt_max=5e-5, max_reisedistanz=1e30, f2_f1=0.5,
          sigma11_22=1.0, sigma11_12=1.0, eps22_11=1.0, eps12_11=1.0)
C3 = dict(C2, N1=1048576, N2=1048576, L=2896.0, FFT_samples=2048, lambda_kapillar=256.0, f2_f1=1.0)


def ensemble(n_runs, seed=2024):
    """Batched ensemble: per-species N log-uniform in [512, 65536], L for an
    area fraction of 0.2, mesh the power of two nearest L/2 in [64, 512],
    NGP/CIC/TSC round-robin, lambda = L/8, dt = 5e-5."""
    rng = np.random.default_rng(seed)
    runs = []
    for r in range(n_runs):
        n = int(round(math.exp(rng.uniform(math.log(512), math.log(65536)))))
        L = math.sqrt(2 * n * math.pi / (4 * 0.2))
        z = min(max(2 ** int(round(math.log2(L / 2))), 64), 512)
        runs.append(dict(C2, N1=n, N2=n, L=L, densGrid_Schema=r % 3, FFT_samples=z,
                         lambda_kapillar=L / 8, f2_f1=1.0))
    return runs


def start_positions(p, seed, dmin=0.8):
    """Seeded uniform positions, pairs closer than dmin re-drawn, in the
    reference layout (cell floor(x/B), offset x - cell*B)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    L = p["L"]
    N = p["N1"] + p["N2"]
    pts = rng.uniform(0, L, (N, 2))
    for _ in range(200):
        tree = cKDTree(pts, boxsize=L)
        pairs = tree.query_pairs(dmin, output_type="ndarray")
        if len(pairs) == 0:
            break
        bad = np.unique(pairs[:, 1])
        pts[bad] = rng.uniform(0, L, (len(bad), 2))
    pts = np.mod(pts, L)
    C = int(math.floor(L / 2 ** (1 / 6)))
    B = L / C
    git = np.minimum(np.floor(pts / B).astype(np.int32), C - 1)
    rel = pts - git * B
    n1 = p["N1"]
    return {0: (git[:n1].copy(), rel[:n1].copy()), 1: (git[n1:].copy(), rel[n1:].copy())}


def alg_bytes(p, stage):
    """Compulsory bytes one launch of a stage moves for one run: every array
    it must read once and write once (particle records 16 B, mesh grids in
    their stored widths, cell tables 4 B per cell)."""
    N = p["N1"] + p["N2"]
    Z = p["FFT_samples"]
    C = int(math.floor(p["L"] / 2 ** (1 / 6)))
    return {
        "deposit": 16 * N + 4 * Z * Z,
        "fft_rows_fwd": 4 * Z * Z + 4 * Z * Z,
        "fft_cols_green": 4 * Z * Z + 2 * Z * Z + 8 * Z * Z,
        "fft_rows_inv": 8 * Z * Z + 8 * Z * Z,
        "particles": 16 * N + 8 * Z * Z + 16 * N + 8 * N,
        # counts read and cleared, start written
        "scan": 4 * C * C + 4 * C * C + 4 * C * C,
        "scatter": 8 * N + 16 * N + 16 * N,
        "reserved7": 0,
        "reserved8": 0,
    }[stage]


def step_bytes(p):
    """Algorithmic bytes of one step: 32 B per particle (16 B state read and
    written) + 32 B per mesh point (density, half spectrum, force grid)."""
    return 32 * (p["N1"] + p["N2"]) + 32 * p["FFT_samples"] ** 2


def ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    e = d.get(kernel)
    return e.get("dram_bytes_per_launch") if e else None


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except OSError:
            return out
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        if sm:
            out["sm_mhz"] = statistics.median(sm)
            out["sm_max_mhz"] = max(mx) if mx else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for k, name in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(name)
        out["reasons"] = sorted(reasons)
        out["samples"] = len(rows)
        return out


# ---------------------------------------------------------------------------
# distributed plumbing (torch.distributed over NCCL: barrier + max of times)

def dist_setup(n):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, ws, local


def _reduce(x, ws, op):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=op)
    return float(t.item())


def dist_max(x, ws):
    import torch.distributed as dist
    return _reduce(x, ws, dist.ReduceOp.MAX) if ws > 1 else x


def dist_sum(x, ws):
    import torch.distributed as dist
    return _reduce(x, ws, dist.ReduceOp.SUM) if ws > 1 else x


def shard(items, rank, ws):
    """Runs of the ensemble this rank steps (round-robin over ranks)."""
    return [(k, q) for k, q in enumerate(items) if k % ws == rank]


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# GPU arm

def flusher(local):
    import torch
    buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:%d" % local)
    return buf


def timed_steps_flushed(run, K, local, buf):
    """K fused steps (one graph launch each), the L2 flushed before every
    step, CUDA events around each step on the library's stream."""
    import torch
    stream = torch.cuda.ExternalStream(run.stream(), device="cuda:%d" % local)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    torch.cuda.synchronize()
    run.sync()
    with torch.cuda.stream(stream):
        for k in range(K):
            buf.fill_(float(k))
            evs[k][0].record(stream)
            run.zeitschritt(1.0)
            evs[k][1].record(stream)
    stream.synchronize()
    run.sync()
    return sum(a.elapsed_time(b) for a, b in evs) / 1e3


def fused_profile(run, K, local, buf):
    """Phase times of the fused step (ms per step), L2 flushed before each
    step; None when the run steps with the stage kernels."""
    import torch
    stream = torch.cuda.ExternalStream(run.stream(), device="cuda:%d" % local)
    acc = None
    for k in range(K):
        with torch.cuda.stream(stream):
            buf.fill_(float(k))
        ph = run.fused_phase_times(1)
        if ph is None:
            return None
        acc = ph if acc is None else {s: acc[s] + ph[s] for s in ph}
    return {s: v / K for s, v in acc.items()}


def stage_profile(run, K, local, buf):
    """Per-stage device times (ms per step) with the L2 flushed before each step."""
    import torch
    stream = torch.cuda.ExternalStream(run.stream(), device="cuda:%d" % local)
    acc = None
    for k in range(K):
        with torch.cuda.stream(stream):
            buf.fill_(float(k))
        st = run.stage_times(1)
        acc = st if acc is None else {s: acc[s] + st[s] for s in st}
    return {s: v / K for s, v in acc.items()}


WORKLOADS = {
    "medium": (C2, "single run, medium: L=512, N1=N2=32768, TSC 512^2, lambda=64, Gamma=1, "
                   "q2=0.5, D=1, dt=5e-5", "c2"),
    "large": (C3, "single run, large: L=2896, N1=N2=2^20, TSC 2048^2, lambda=256, Gamma=1, "
                  "q1=q2=1, D=1, dt=5e-5", "c3"),
}
NOISE = "uniform disk of radius sqrt(5) (the reference's noise, dynamik_methoden.cpp:1317-1339)"


def workload_config(name):
    """The `config` object both arms print for a workload (identical keys)."""
    base, wl, _ = WORKLOADS[name]
    return {"workload": wl, "particles": base["N1"] + base["N2"], "mesh": base["FFT_samples"],
            "noise": NOISE}


def gpu_arm(args):
    import torch
    import bdsim
    rank, ws, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    buf = flusher(local)
    peak, peak_kind = measured_peaks()
    base, wl_name, _ = WORKLOADS[args.workload]
    p = dict(base, noise_kind=bdsim.NOISE_DISK)
    N = p["N1"] + p["N2"]
    K, W = args.steps, args.warmup
    start = start_positions(p, 1000 + rank)
    run = bdsim.Run(p, seed=1 + rank, device=local)
    run.set_positions_all(start)
    run.zeitschritte(W)
    barrier(ws)
    with Clocks(local) as ck:
        t_dev = timed_steps_flushed(run, K, local, buf)
    t_dev = dist_max(t_dev, ws)
    value = ws * N * K / t_dev
    launches = run.launches_per_step() * K
    # roofline. Fused step: the one kernel is the whole step (its launch
    # time is the event-timed step), its phases from device timestamps.
    # Stage kernels: the dominant stage, algorithmic bytes / its event time.
    phases = fused_profile(run, min(K, 200), local, buf)
    if phases is not None:
        dom = "k_fused (whole step in one cooperative launch)"
        achieved = step_bytes(p) / (t_dev / K) / 1e9
        stages = None
    else:
        stages = stage_profile(run, min(K, 200), local, buf)
        dom = max(stages, key=stages.get)
        achieved = alg_bytes(p, dom) / (stages[dom] * 1e-3) / 1e9
    # e2e through the C ABI with host buffers
    run2 = bdsim.Run(p, seed=1 + rank, device=local)
    # the caller's output arrays, allocated and written once before the timed
    # region (np.zeros maps its pages lazily: the first write would time the
    # operating system's page faults, not the copy)
    host_out = {s: (np.zeros((p["N%d" % (s + 1)], 2), np.int32), np.zeros((p["N%d" % (s + 1)], 2))) for s in (0, 1)}
    for s in (0, 1):
        host_out[s][0].fill(0)
        host_out[s][1].fill(0.0)
    run2.set_positions_all(start)
    run2.zeitschritte(W)
    run2.sync()
    # E2E_REPS repetitions of the whole call sequence (a few ms each, host
    # wall clock): the median, max over ranks
    t_reps = []
    for _ in range(E2E_REPS):
        run2.sync()
        barrier(ws)
        t0 = time.perf_counter()
        run2.set_positions_all(start)
        for _ in range(K):
            run2.zeitschritt(1.0)
        run2.get_positions(host_out)
        t_reps.append(dist_max(time.perf_counter() - t0, ws))
    t_e2e = statistics.median(t_reps)
    e2e = ws * N * K / t_e2e
    extras = {}
    if not args.no_extras:
        extras = extras_gpu(args, rank, ws, local, buf, peak)
    res = None
    if rank == 0:
        res = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": ws, "steps": K,
            "warmup": W, "ms_per_step": 1e3 * t_dev / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic: seeded uniform positions, pairs < 0.8 sigma re-drawn",
            "config": workload_config(args.workload),
            "parallelism": "replicas x%d" % ws,
            "l2": "flushed (256 MB write) before every timed step",
            "timing": "CUDA events on the library stream, summed per step, max over ranks",
            "e2e": {"value": e2e, "unit": "particle-steps/s", "h2d_bytes_per_step": 16 * N / K,
                    "d2h_bytes_per_step": 16 * N / K,
                    "calls": "bd_set_positions_all, %d x bd_zeitschritt, bd_get_positions_all" % K,
                    "timing": "host wall clock, median of %d repetitions, max over ranks" % E2E_REPS},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": ncu_traffic(dom),
                         "step_alg_bytes": step_bytes(p),
                         "step_frac": step_bytes(p) / (t_dev / K) / 1e9 / peak},
            "clocks": ck.summary(),
        }
        if phases is not None:
            res["roofline"]["phase_ms"] = phases
        else:
            res["roofline"]["stage_ms"] = stages
        res.update(extras)
    return res, rank, ws


E2E_REPS = 5  # repetitions of the headline's end-to-end call sequence

C1 = dict(C2, N1=1000, N2=1000, L=100.0, densGrid_Schema=1, FFT_samples=128, lambda_kapillar=10.0,
          dt_max=1e-4, f2_f1=1.0)


def tune_record(tune):
    """The batch autotuner's choices (bd_tune_result) for the JSON line."""
    return {"fft_items_min": tune.fft_items_min, "dep_tiles_min": tune.dep_tiles_min,
            "candidates": tune.candidates, "default_mesh_ms": tune.default_ms, "best_mesh_ms": tune.best_ms,
            "particle_shape": ["four CTAs per SM", "five CTAs per SM"][tune.particle_shape],
            "default_particle_ms": tune.particle_default_ms, "best_particle_ms": tune.particle_best_ms}


def extras_gpu(args, rank, ws, local, buf, peak):
    import bdsim
    out = {}
    # plain small run (L=100, N1=N2=1000, CIC 128^2, dt=1e-4), its 1000 steps
    p1 = dict(C1, noise_kind=bdsim.NOISE_DISK)
    r1 = bdsim.Run(p1, seed=11 + rank, device=local)
    r1.set_positions_all(start_positions(p1, 2000 + rank))
    r1.zeitschritte(args.warmup)
    K1 = args.small_steps
    t1 = dist_max(timed_steps_flushed(r1, K1, local, buf), ws)
    out["plain_small"] = {"value": ws * (p1["N1"] + p1["N2"]) * K1 / t1, "unit": "particle-steps/s",
                          "steps": K1, "ms_per_step": 1e3 * t1 / K1,
                          "step_frac": step_bytes(p1) / (t1 / K1) / 1e9 / peak,
                          "gpu_launches": r1.launches_per_step() * K1,
                          "config": "L=100, N1=N2=1000, CIC 128^2, lambda=10, dt=1e-4, uniform-disk noise",
                          "l2": "flushed before every timed step"}
    r1.close()
    # batched ensemble: runs partitioned across ranks
    runs = ensemble(args.ensemble_runs)
    mine = shard(runs, rank, ws)
    b = bdsim.Batch([dict(q, noise_kind=bdsim.NOISE_DISK) for _, q in mine],
                    [5000 + k for k, _ in mine], device=local)
    Kb = args.batch_steps
    b.step(args.warmup)
    # the plan autotuner (transform items per launch), then warm up again
    tune = b.autotune(3)
    b.step(args.warmup)
    b.sync()
    import torch
    stream = torch.cuda.ExternalStream(b.stream(), device="cuda:%d" % local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(ws)
    e0.record(stream)
    b.step(Kb)
    e1.record(stream)
    b.sync()
    t = dist_max(e0.elapsed_time(e1) / 1e3, ws)
    n_tot = sum(q["N1"] + q["N2"] for q in runs)
    bytes_tot = sum(step_bytes(q) for q in runs)
    out["batched"] = {"value": n_tot * Kb / t, "unit": "particle-steps/s", "runs": len(runs),
                      "particles": n_tot, "steps": Kb, "ms_per_step": 1e3 * t / Kb,
                      "step_alg_bytes": bytes_tot, "step_frac": bytes_tot / (t / Kb) / 1e9 / peak,
                      "gpu_launches": b.launches_per_step() * Kb,
                      "l2": "working set %.0f MB > L2" % (bytes_tot / 1e6),
                      "autotune": tune_record(tune)}
    ph = b.phase_times(5)
    if ph is not None:
        out["batched"]["phase_ms"] = ph
    else:
        out["batched"]["stage_ms"] = b.stage_times(5)
    b.close()
    # large single run (replica per rank), its 2000 steps
    p3 = dict(C3, noise_kind=bdsim.NOISE_DISK)
    r3 = bdsim.Run(p3, seed=3 + rank, device=local)
    r3.zeitschritte(args.warmup)
    K3 = args.large_steps
    t3 = dist_max(timed_steps_flushed(r3, K3, local, buf), ws)
    out["plain_large"] = {"value": ws * (p3["N1"] + p3["N2"]) * K3 / t3, "unit": "particle-steps/s",
                          "steps": K3, "ms_per_step": 1e3 * t3 / K3,
                          "step_frac": step_bytes(p3) / (t3 / K3) / 1e9 / peak,
                          "gpu_launches": r3.launches_per_step() * K3}
    ph = fused_profile(r3, 5, local, buf)
    if ph is not None:
        out["plain_large"]["phase_ms"] = ph
    else:
        out["plain_large"]["stage_ms"] = stage_profile(r3, 5, local, buf)
    r3.close()
    # served stream below capacity (rank 0 of each node serves its own stream)
    out["served"] = serve_bench(local, args.serve_rate, args.serve_seconds, args.serve_scale, args.serve_tick)
    return out


def serve_requests(rate, seconds, scale, seed=77):
    """Poisson arrivals at `rate`/s for `seconds` s; N1=N2 log-uniform in
    [1024, 262144] (the serving workload's sizes), steps log-uniform in
    [1e3, 1e5] times `scale`, L for an area fraction of 0.2, mesh the power of
    two nearest L/2 in [64, 512], CIC or TSC alternating, lambda = L/8."""
    import bdsim
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            break
        n = int(round(math.exp(rng.uniform(math.log(1024), math.log(262144)))))
        steps = int(round(math.exp(rng.uniform(math.log(1e3), math.log(1e5))) * scale))
        steps = max(steps, 10)
        L = math.sqrt(2 * n * math.pi / (4 * 0.2))
        z = min(max(2 ** int(round(math.log2(L / 2))), 64), 512)
        p = dict(C2, N1=n, N2=n, L=L, densGrid_Schema=1 + (len(reqs) % 2), FFT_samples=z,
                 lambda_kapillar=L / 8, f2_f1=1.0, noise_kind=bdsim.NOISE_DISK)
        reqs.append((t, p, steps))
    return reqs


def serve_bench(local, rate, seconds, scale, tick):
    """The served stream of serve_requests(rate, seconds, scale), snapshots
    every 1000 steps; requests are submitted at their arrival times (wall
    clock) and the server ticks meanwhile. Returns throughput (particle-steps
    completed / wall time), p50/p99 completion latency and the offered load."""
    import bdsim
    reqs = serve_requests(rate, seconds, scale)
    srv = bdsim.Server(device=local, steps_per_tick=tick)
    t0 = time.perf_counter()
    ids = []
    k = 0
    open_ids = set()
    while k < len(reqs) or open_ids:
        now = time.perf_counter() - t0
        while k < len(reqs) and reqs[k][0] <= now:
            rid = srv.submit(reqs[k][1], 900 + k, reqs[k][2], snapshot_every=1000)
            ids.append(rid)
            open_ids.add(rid)
            k += 1
        active = srv.tick()
        open_ids = {i for i in open_ids if srv.poll(i).state < 2}
        if active == 0 and k < len(reqs):
            time.sleep(max(0.0, min(0.01, reqs[k][0] - (time.perf_counter() - t0))))
    st = srv.stats()
    wall = time.perf_counter() - t0
    offered = sum(2 * q[1]["N1"] * q[2] for q in reqs) / seconds
    out = {"value": st.particle_steps / wall, "unit": "particle-steps/s", "requests": len(reqs),
           "offered_particle_steps_per_s": offered,
           "completed": st.completed, "p50_latency_s": st.p50_latency_s,
           "p99_latency_s": st.p99_latency_s, "max_latency_s": st.max_latency_s, "wall_s": wall,
           "step_s": st.step_s, "host_s": st.host_s, "admit_s": st.admit_s, "plan_s": st.plan_s,
           "fetch_s": st.fetch_s,
           "arrivals": "Poisson %g/s for %g s" % (rate, seconds), "steps_scale": scale,
           "steps_per_tick": tick}
    srv.close()
    return out


def batched_arm(args):
    """--workload batched: the 256-run ensemble as the line's workload (runs
    partitioned across ranks): K steps of every run, CUDA events on the
    batch's stream (working set above L2), the plan autotuned first; e2e
    through the batch C ABI with host buffers (bd_batch_set_positions_all of
    every run, bd_batch_step(K), bd_batch_get_positions_all of every run)."""
    import torch
    import bdsim
    rank, ws, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    peak, peak_kind = measured_peaks()
    runs = ensemble(args.ensemble_runs)
    mine = shard(runs, rank, ws)
    params = [dict(q, noise_kind=bdsim.NOISE_DISK) for _, q in mine]
    b = bdsim.Batch(params, [5000 + k for k, _ in mine], device=local)
    K, W = args.steps, args.warmup
    b.step(W)
    tune = b.autotune(3)
    b.step(W)
    b.sync()
    stream = torch.cuda.ExternalStream(b.stream(), device="cuda:%d" % local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(ws)
    with Clocks(local) as ck:
        e0.record(stream)
        b.step(K)
        e1.record(stream)
        b.sync()
    t = dist_max(e0.elapsed_time(e1) / 1e3, ws)
    n_tot = sum(q["N1"] + q["N2"] for q in runs)
    bytes_tot = sum(step_bytes(q) for q in runs)
    ph = b.phase_times(5)
    # e2e: host positions in, K steps, host positions out
    host = [b.get_positions(k) for k in range(len(params))]
    b.sync()
    barrier(ws)
    t0 = time.perf_counter()
    for k in range(len(params)):
        b.set_positions(k, host[k])
    b.step(K)
    host = [b.get_positions(k) for k in range(len(params))]
    t_e2e = dist_max(time.perf_counter() - t0, ws)
    nbytes = sum(24 * (q["N1"] + q["N2"]) for q in params)
    res = None
    if rank == 0:
        res = {"metric": METRIC, "value": n_tot * K / t, "unit": "particle-steps/s", "n_gpus": ws, "steps": K,
               "warmup": W, "ms_per_step": 1e3 * t / K, "higher_is_better": True, "scaling": "strong",
               "vs_baseline": None, "dtype": "fp32", "data": "synthetic: seeded uniform positions per run",
               "config": {"workload": "batched ensemble: 256 runs, N per species log-uniform in [512, 65536], "
                                      "area fraction 0.2, meshes 64^2-256^2, NGP/CIC/TSC round-robin, "
                                      "lambda=L/8, dt=5e-5", "runs": len(runs), "particles": n_tot,
                          "noise": NOISE},
               "parallelism": "runs partitioned over %d rank(s)" % ws,
               "l2": "working set %.0f MB > L2" % (bytes_tot / 1e6),
               "timing": "CUDA events on the batch stream around K steps, max over ranks",
               "e2e": {"value": n_tot * K / t_e2e, "unit": "particle-steps/s",
                       "h2d_bytes_per_step": nbytes / K, "d2h_bytes_per_step": nbytes / K,
                       "calls": "bd_batch_set_positions_all (every run), bd_batch_step(%d), "
                                "bd_batch_get_positions_all (every run)" % K},
               "gpu_launches": b.launches_per_step() * K,
               "roofline": {"bound": "hbm", "kernel": "whole step (%d launches)" % b.launches_per_step(),
                            "achieved": bytes_tot / (t / K) / 1e9, "peak": peak, "peak_source": peak_kind,
                            "unit": "GB/s", "frac": bytes_tot / (t / K) / 1e9 / peak, "traffic": None,
                            "step_alg_bytes": bytes_tot},
               "autotune": tune_record(tune),
               "clocks": ck.summary()}
        if ph is not None:
            res["roofline"]["phase_ms"] = ph
    b.close()
    return res, rank, ws


def served_arm(args):
    """--workload served: the serving workload as stated (Poisson 50/s for
    60 s, unscaled step counts), one JSON line with p50/p99."""
    import torch
    rank, ws, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    peak, _ = measured_peaks()
    with Clocks(local) as ck:
        res = serve_bench(local, 50.0, 60.0, 1.0, args.serve_tick)
    line = {"metric": METRIC, "value": res["value"], "unit": "particle-steps/s", "n_gpus": 1,
            "steps": None, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32", "data": "synthetic: Poisson request stream from a seed",
            "config": {"workload": "served: Poisson 50/s for 60 s, N1=N2 log-uniform in [1024, 262144], "
                                   "steps log-uniform in [1e3, 1e5], CIC or TSC, lambda=L/8, "
                                   "snapshots every 1000 steps", "noise": NOISE},
            "served": res, "clocks": ck.summary()}
    return line, rank, ws


# ---------------------------------------------------------------------------
# CPU legs: the compiled reference (oracle/_ref/c2/bdref) or the oracle port

def host_cpu():
    """The host CPU model (first "model name" of /proc/cpuinfo), for the
    CPU baseline's record."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except (OSError, ValueError):
        pass
    return "unknown"


def cpu_reference(p, steps, warmup, procs, build="c2"):
    """Time zeitschritt() of the reference's own code on `procs` host cores
    at once (one independent run per process: the reference is single
    threaded, maxThreads = 1 in parameter.h:93). Returns particle-steps/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    exe = oracle.ref_exe(build)
    N = p["N1"] + p["N2"]
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "start.pos")
        oracle.write_pos(f, start_positions(p, 1000))
        files = [f] * procs
        if os.path.exists(exe):
            t0 = time.perf_counter()
            ps = [subprocess.Popen([exe, "timefile", files[k], str(steps), str(warmup)], cwd=d,
                                   stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                  for k in range(procs)]
            outs = [q.communicate()[0] for q in ps]
            wall = time.perf_counter() - t0
            secs = [json.loads([l for l in o.splitlines() if l.startswith("{")][0])["seconds"] for o in outs]
            kind = "reference"
        else:
            import multiprocessing as mp
            ctx = mp.get_context("spawn")
            with ctx.Pool(procs) as pool:
                secs = pool.starmap(_oracle_time, [(p, files[k], steps, warmup) for k in range(procs)])
            kind = "port"
    # every process times its own steps; aggregate over the slowest
    return procs * N * steps / max(secs), kind, max(secs)


def _oracle_time(p, path, steps, warmup):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import configs
    import oracle
    q = dict(configs.param_defaults())
    q.update(p)
    o = oracle.Oracle(q, 12345)
    o.set_positions(oracle.read_pos(path))
    o.step(warmup)
    t0 = time.perf_counter()
    o.step(steps)
    return time.perf_counter() - t0


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    if args.workload == "served":
        return {"impl": "reference", "unavailable": "the reference has no serving mode (its runs loop, "
                                                    "main.cpp:130, steps one run at a time); its CPU rate "
                                                    "is the medium workload's reference line"}
    if args.workload == "batched":
        return {"impl": "reference", "unavailable": "the reference compiles one parameter set into its binary "
                                                    "(parameter.h), so the ensemble's 256 parameter sets are "
                                                    "256 builds; its CPU rate is the medium workload's "
                                                    "reference line"}
    base, wl_name, build = WORKLOADS[args.workload]
    procs = min(os.cpu_count() or 1, args.ref_procs)
    steps = max(1, min(args.steps, args.ref_steps))
    value, kind, secs = cpu_reference(dict(base), steps, args.warmup, procs, build)
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp64", "data": "synthetic: seeded uniform positions, pairs < 0.8 sigma re-drawn",
        "config": workload_config(args.workload),
        "parallelism": "%d independent runs, one per core" % procs,
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": procs, "kind": kind,
                         "cpu": host_cpu(),
                         "sample": "%d steps (+%d warm-up) of the single-run workload in each of %d "
                                   "processes; reference built with g++ -O3 and the project FFT shim "
                                   "(FFTW unavailable)" % (steps, args.warmup, procs)},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="medium", choices=sorted(WORKLOADS) + ["batched", "served"])
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ensemble-runs", type=int, default=256)
    ap.add_argument("--small-steps", type=int, default=1000)
    ap.add_argument("--batch-steps", type=int, default=5000)
    ap.add_argument("--large-steps", type=int, default=2000)
    ap.add_argument("--serve-rate", type=float, default=1.0,
                    help="arrivals per second of the served extra (below the server's capacity)")
    ap.add_argument("--serve-seconds", type=float, default=20.0)
    ap.add_argument("--serve-scale", type=float, default=1.0,
                    help="factor on the served requests' step counts")
    ap.add_argument("--serve-tick", type=int, default=100)
    ap.add_argument("--ref-procs", type=int, default=64)
    ap.add_argument("--ref-steps", type=int, default=40)
    ap.add_argument("--cpu-steps", type=int, default=40)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        res = reference_arm(args)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    if args.workload in ("served", "batched"):
        res, rank, ws = (served_arm if args.workload == "served" else batched_arm)(args)
        if rank == 0:
            print(json.dumps(res), flush=True)
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    res, rank, ws = gpu_arm(args)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        base, _, build = WORKLOADS[args.workload]
        procs = min(os.cpu_count() or 1, args.ref_procs)
        v, kind, secs = cpu_reference(dict(base), args.cpu_steps, 2, procs, build)
        res["cpu_baseline"] = {"value": v, "unit": "particle-steps/s", "cores": procs, "kind": kind,
                               "cpu": host_cpu(),
                               "sample": "%d steps (+2 warm-up) of the single-run workload in each of %d "
                                         "processes (%.1f s per process)" % (args.cpu_steps, procs, secs)}
    if rank == 0:
        print(json.dumps(res), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
