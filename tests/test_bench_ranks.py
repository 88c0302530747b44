"""The multi-rank plumbing of bench.py (replicas: barrier and max-over-ranks
timing, no data-path collective) on two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_init()
    assert (w, r, local) == (ws, rank, rank)
    bench.barrier(w)
    out[rank] = bench.max_over_ranks(1.5 + rank, w)   # each rank's "elapsed ms"
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_rank_max_over_ranks_and_barrier():
    ws, port = 2, _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(ws, port, out), nprocs=ws, join=True)
        assert dict(out) == {0: 2.5, 1: 2.5}
