"""The multi-GPU form of the stepping path is replicas: each rank steps its
own batch, with no collective on the data path; the benchmark combines the
ranks' results with two host-side reductions (max of the device time, sum of
the particle-steps).  Checked here with two gloo ranks on the CPU, through
the benchmark's own functions."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, queue):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r stepped 1000 * (r + 1) particle-steps in 10 * (r + 1) ms
        steps, ms = 1000 * (rank + 1), 10.0 * (rank + 1)
        value, ms_max, units = bench.replica_rate(steps, ms, world)
        bench.barrier(world)
        queue.put((rank, value, ms_max, units, bench.max_over_ranks(float(rank), world)))
    finally:
        dist.destroy_process_group()


def test_replica_rate_over_two_gloo_ranks():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, value, ms_max, units, mx in res:
        assert units == 3000            # 1000 + 2000 particle-steps
        assert ms_max == 20.0           # the slower rank
        assert value == pytest.approx(3000 / 0.020)
        assert mx == 1.0


def test_replica_rate_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    value, ms_max, units = bench.replica_rate(500, 5.0, 1)
    assert (value, ms_max, units) == (pytest.approx(1e5), 5.0, 500)
