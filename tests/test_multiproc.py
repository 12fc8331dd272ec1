"""The multi-GPU (replicas-only) host logic of bench.py on CPU ranks: two
gloo processes rendezvous on 127.0.0.1, seed their replicas differently and
agree on the max-over-ranks time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import bench
    import torch.distributed as dist
    ws, r, _ = bench.dist_init("gloo")
    seed = bench.replica_seed(2, r)
    t = bench.reduce_max(1.0 + r * 0.5, ws)
    bench.barrier(ws)
    q.put((r, ws, seed, t))
    dist.destroy_process_group()


def test_two_gloo_replicas_agree_on_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [r[1] for r in res] == [2, 2]
    assert [r[2] for r in res] == [2, 3]          # distinct seeded replicas
    assert all(r[3] == 1.5 for r in res)          # max over ranks
