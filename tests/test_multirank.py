"""The replica (multi-rank) plumbing of bench.py on CPU: two gloo ranks, the
max-over-ranks timing reduction and the whole-job rate it feeds."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import bench
    w, r, local = bench.dist_env()
    dist = bench.dist_init(w, local, backend="gloo")
    ms = 10.0 * (rank + 1)  # rank 1 is the slow replica
    bench.barrier(dist)
    ms_max = bench.dist_max(dist, ms, local)
    out[rank] = (ms_max, bench.whole_job_rate(w, 1_000_000, 100, ms_max))
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    ws, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    assert res[0] == res[1]
    ms_max, rate = res[0]
    assert ms_max == pytest.approx(20.0)
    assert rate == pytest.approx(2 * 1e6 * 100 / 20e-3 / 1e9)
