"""The N>1 bench path on CPU: two gloo ranks, each a replica with its own box."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from ct2_b200 import ics, replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    # each replica has its own seeded box (seed + rank), as bench.py does
    box = ics.plummer_spheres(1000 + 500 * rank, seed=rank, nspheres=2, a=0.05)
    ms = 10.0 + 5.0 * rank
    value, ms_max = replicas.job_throughput(len(box["x"]), ms)
    out[rank] = (value, ms_max, int(box["x"][0]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_gloo():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True,
                       start_method="spawn")
    v0, m0, x0 = out[0]
    v1, m1, x1 = out[1]
    # the slowest rank bounds the job, every rank reports the same figures
    assert m0 == m1 == 15.0
    assert v0 == v1 == pytest.approx((1000 + 1500) / 15e-3)
    # and the replicas integrated different boxes
    assert x0 != x1


def test_single_process_is_identity():
    from ct2_b200 import replicas
    v, ms = replicas.job_throughput(2048, 4.0)
    assert ms == 4.0 and v == pytest.approx(2048 / 4e-3)
