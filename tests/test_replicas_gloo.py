"""The multi-GPU path (one replica per GPU, MAX-over-ranks timing) on CPU with
two gloo ranks: every rank sees the slowest rank's time and the same
whole-job throughput; seeds differ per rank."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from hackathon_b200 import replicas as R
    ms = [3.0, 5.0][rank]  # rank 1 is the slow one
    m = R.max_over_ranks(ms, dist)
    out[rank] = (m, R.weak_scaling_throughput(1024, m, world), R.rank_seed(1, rank))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_time_and_throughput():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == 5.0
    assert res[0][1] == res[1][1] == pytest.approx(2 * 1024 / 5e-3)
    assert res[0][2] != res[1][2]


def test_single_process_is_identity():
    from hackathon_b200 import replicas as R
    assert R.max_over_ranks(2.5) == 2.5
    assert R.weak_scaling_throughput(1024, 4.0, 1) == pytest.approx(256000.0)
