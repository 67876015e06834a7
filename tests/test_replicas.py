"""The multi-GPU mode's rank bookkeeping (alea_b200.replicas) on CPU: two
gloo ranks, as bench.py runs one replica per GPU under torchrun.  Each rank
has its own seed; the job's time is the slowest rank's and its work the sum
of the ranks'; nothing else crosses ranks."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from alea_b200.replicas import Replicas, replica_seed
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r = Replicas(dist, torch.device("cpu"))
        ms = 10.0 + 5.0 * rank          # rank 1 is the slower one
        moves = 1000.0 * (rank + 1)
        r.barrier()
        out[rank] = dict(seed=replica_seed(20261203, rank), world=r.world, rank=r.rank,
                         ms=r.max(ms), moves=r.sum(moves), rate=r.throughput(moves, ms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_the_bench():
    import torch.multiprocessing as mp
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = [dict(out[i]) for i in range(2)]
    assert res[0]["seed"] != res[1]["seed"]
    for i, r in enumerate(res):
        assert r["world"] == 2 and r["rank"] == i
        assert r["ms"] == 15.0 and r["moves"] == 3000.0          # max time, summed work
        assert r["rate"] == pytest.approx(3000.0 / 15e-3)


def test_single_replica_without_a_process_group():
    from alea_b200.replicas import Replicas
    r = Replicas(None)
    r.barrier()
    assert (r.world, r.rank) == (1, 0)
    assert r.max(3.0) == 3.0 and r.sum(4.0) == 4.0 and r.throughput(10.0, 2.0) == 5000.0
