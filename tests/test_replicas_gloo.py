"""The multi-GPU bench runs independent replicas (one process per GPU, no collective on the data
path); its only cross-rank steps are the max/min reductions of the timings. Exercised here with
two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # rank r "took" 10 + r ms for its steps and 3 - r ms end to end
    ms, other = bench._over_ranks([10.0 + rank, 3.0 - rank], "max", dist, "cpu")
    lo = bench._over_ranks([3.0 - rank], "min", dist, "cpu")[0]
    out[rank] = (ms, other, lo, bench._job_throughput(world, 4096 * 100, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reductions_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1]
    ms, other, lo, value = res[0]
    assert ms == 11.0 and other == 3.0 and lo == 2.0
    assert value == pytest.approx(2 * 4096 * 100 / 11e-3)


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench._over_ranks([1.5, 2.5], "max", None, "cpu") == [1.5, 2.5]
