"""Multi-rank plumbing of bench.py on CPU: world_size 2 over gloo. Ranks shard
the ensemble without overlap and agree on the max/sum of their timings."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    runs = bench.ensemble(16, seed=3)
    mine = [k for k, _ in bench.shard(runs, rank, ws)]
    t = bench.dist_max(1.0 + rank, ws)
    n = bench.dist_sum(float(sum(runs[k]["N1"] + runs[k]["N2"] for k in mine)), ws)
    bench.barrier(ws)
    dist.destroy_process_group()
    q.put((rank, mine, t, n))


def test_two_ranks_shard_and_reduce():
    import multiprocessing as mp
    import socket
    sys.path.insert(0, ROOT)
    import bench
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    out.sort()
    runs = bench.ensemble(16, seed=3)
    a, b = out[0][1], out[1][1]
    assert sorted(a + b) == list(range(16)) and not set(a) & set(b)
    assert out[0][2] == out[1][2] == 2.0
    total = sum(r["N1"] + r["N2"] for r in runs)
    assert out[0][3] == out[1][3] == pytest.approx(total)
