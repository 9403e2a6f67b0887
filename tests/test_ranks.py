"""The N>1 path of bench.py on CPU processes: two gloo ranks run the same
barrier / max-over-ranks / whole-job aggregation logic as the NCCL ranks of a
multi-GPU run (replicas only: no collective on the data path)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys

    sys.path.insert(0, os.path.join(HERE, ".."))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import bench

    r = bench.Ranks(world, backend="gloo")
    try:
        r.barrier()
        own_ms = 10.0 * (rank + 1)  # each rank's own device time
        ms = r.max(own_ms)
        out[rank] = (r.world, r.rank, ms, r.throughput(1000, 5, ms))
    finally:
        r.close()


def test_two_gloo_ranks_barrier_max_and_aggregate():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(out.keys()) == [0, 1]
    for rank, (w, rk, ms, value) in out.items():
        assert (w, rk) == (2, rank)
        assert ms == pytest.approx(20.0)  # max over ranks, on every rank
        assert value == pytest.approx(2 * 1000 * 5 / 0.020)  # all ranks' cells / max time
