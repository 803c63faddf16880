"""Host logic of the multi-GPU (replica) form on CPU: world_size-2 gloo process groups."""
import importlib
import os
import socket
import sys

import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rep = importlib.import_module("zksync-crypto-gpu_b200.replicas")
    m = rep.max_over_ranks(10.0 + rank)
    jobs = [(12 + (i % 5), 8 * (1 + i % 4), 1 + i % 2) for i in range(11)]
    mine = rep.shard_jobs(jobs, rank, world)
    q.put((rank, m, mine, rep.rank_seed("s", rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reduction_and_sharding():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert out[0][1] == out[1][1] == 11.0  # max over ranks
    jobs = [(12 + (i % 5), 8 * (1 + i % 4), 1 + i % 2) for i in range(11)]
    got = sorted(out[0][2] + out[1][2])
    assert got == sorted(jobs)  # every job on exactly one rank
    assert out[0][3] != out[1][3]  # independent inputs per replica
    rep = importlib.import_module("zksync-crypto-gpu_b200.replicas")
    c0 = sum(rep.job_cost(j) for j in out[0][2])
    c1 = sum(rep.job_cost(j) for j in out[1][2])
    assert max(c0, c1) / min(c0, c1) < 2.0  # balanced


def test_aggregate_rate():
    rep = importlib.import_module("zksync-crypto-gpu_b200.replicas")
    assert rep.aggregate_rate(100.0, 4, 2.0) == 200.0
    assert rep.max_over_ranks(3.5) == 3.5  # no process group: identity
