"""Replica runs on 2 ranks with gloo on CPU: the barrier and the
max-over-ranks reduction the bench uses for its device times."""
from __future__ import annotations

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


def _worker(rank, ws, port, out):
    os.environ.update({"WORLD_SIZE": str(ws), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from eman2_b200 import replicas
    w, r, _ = replicas.init("gloo", timeout_s=60)
    replicas.barrier(w)
    out[r] = (replicas.max_over_ranks(1.5 + r, w), replicas.sum_over_ranks(1.0 + r, w))
    replicas.finalize(w)
    import torch.distributed as dist
    assert not dist.is_initialized()


@pytest.mark.timeout(120)
def test_two_rank_max_and_sum():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(100)
        assert p.exitcode == 0
    assert out[0] == out[1] == (2.5, 3.0)
