"""The multi-GPU plumbing on CPU: two gloo ranks (replicas, no data-path
collective) agree on the barrier and on the max over ranks of their times,
draw distinct frame seeds, and the whole-job rate counts every rank's work
against the slowest rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from vitrum_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r, w, lr = replicas.env_rank()
    g = replicas.Group(w, "gloo", timeout_s=60)
    g.barrier()
    my_time = 1.0 + 0.5 * r
    mx = g.max(my_time)
    seeds = [replicas.replica_seed(r, s) for s in range(3)]
    q.put((r, w, lr, mx, seeds, replicas.whole_job_rate(100.0, w, mx)))
    g.close()


def test_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[3] == 1.5 for o in out)  # max over ranks, seen by every rank
    assert not set(out[0][4]) & set(out[1][4])  # replicas render distinct frames
    assert out[0][5] == pytest.approx(2 * 100.0 / 1.5)


def test_single_process_group_is_inert():
    g = replicas.Group(1)
    g.barrier()
    assert g.max(3.0) == 3.0
    g.close()
