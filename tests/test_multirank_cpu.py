"""The N > 1 path of bench.py on CPU: independent replicas (one per rank, no
data-path collective), timings combined as the maximum over ranks.  Two
`gloo` ranks on 127.0.0.1 stand in for two GPUs; the reduction is the same
call the bench makes under torchrun with NCCL."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as tdist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank's own timings (ms): the slowest rank sets every reported number
        mine = [10.0 + rank, 5.0 - rank, 100.0 * (rank + 1)]
        out[rank] = bench.max_over_ranks(mine)
        tdist.barrier()
    finally:
        tdist.destroy_process_group()


def test_timings_are_the_maximum_over_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(world):
            assert out[r] == [11.0, 5.0, 200.0]


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.5, 2.0]) == [1.5, 2.0]


def test_replica_seeds_differ_per_rank():
    """Each rank advances its own replica: the bench seeds rank r's field with SEED + r."""
    sys.path.insert(0, ROOT)
    import bench
    src = open(os.path.join(ROOT, "bench.py")).read()
    assert "SEED + rank" in src
    assert bench.workload()["parallelism"] == "replicas"


if __name__ == "__main__":
    pytest.main([__file__, "-q"])
