"""The multi-GPU form of the path is replicas (every rank runs the whole workload; no data-path collective).
Its host logic, the whole-job throughput over the slowest rank, runs here on two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    import bench

    # rank r took (r + 1) seconds on the device and 2 (r + 1) end to end for 1e6 units
    value, e2e, td, te = bench.replica_throughput(1e6, float(rank + 1), 2.0 * (rank + 1), world, dist, "cpu")
    out[rank] = (value, e2e, td, te)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_replica_throughput_takes_the_slowest_rank(world):
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        value, e2e, td, te = out[r]
        assert td == float(world) and te == 2.0 * world       # every rank sees the slowest rank's times
        assert value == 1e6 * world / world and e2e == 1e6 * world / (2.0 * world)


def test_single_process_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.replica_throughput(10.0, 2.0, 4.0, 1) == (5.0, 2.5, 2.0, 4.0)
