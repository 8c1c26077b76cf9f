"""Multi-process plumbing of `bench.py --gpus N` (independent replicas), on CPU with gloo:
the barrier, the max-over-ranks of the timings and the whole-job aggregation."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, pg = bench.dist_setup(backend="gloo")
    try:
        bench.barrier(pg)
        ms = bench.max_over_ranks(pg, 10.0 + rank, device="cpu")   # rank r "took" 10 + r ms
        out[rank] = (w, r, ms, bench.whole_job_value(w, 1000, 5, ms))
        bench.barrier(pg)
    finally:
        pg.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_replica_timing_is_max_over_ranks(world):
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == list(range(world))
    for r, (w, rr, ms, value) in res.items():
        assert (w, rr) == (world, r)
        assert ms == 10.0 + world - 1                  # the slowest rank sets the time
        assert value == pytest.approx(world * 1000 * 5 / (ms / 1e3) / 1e6)
