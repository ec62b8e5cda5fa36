"""Replica-mode plumbing with world_size 2 on the gloo backend (CPU): frame
assignment covers the orbit exactly once per period, max/sum over ranks, and
the barrier; plus a rank that fails is seen by the other rank as an error of
its next collective (short process-group timeout), not as a hang."""
import os
import socket
import sys

import pytest

import helpers


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, queue, fail_rank):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(helpers.ROOT, "tests"))
    import helpers as h

    h.package()
    import ve_b200.dist as vd

    try:
        dist = vd.init("gloo", timeout_s=20.0)
        frames = vd.frame_assignment(8, rank, world, 64)
        t = vd.max_over_ranks(1.0 + rank, dist)
        n = vd.sum_over_ranks(100 * (rank + 1), dist)
        vd.barrier(dist)
        if fail_rank == rank:
            os._exit(3)  # leaves between steps, no collective in flight
        err = None
        if fail_rank is not None:
            try:
                vd.sum_over_ranks(1.0, dist)
            except Exception as e:  # the peer is gone: the collective errors out
                err = type(e).__name__
        queue.put((rank, frames, t, n, err))
        if fail_rank is None:
            vd.shutdown(dist)
    except Exception as e:  # pragma: no cover - reported to the parent
        queue.put((rank, "error", repr(e), None, None))


def _run(world, fail_rank=None):
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    expected = world - (1 if fail_rank is not None else 0)
    for _ in range(expected):
        r = q.get(timeout=120)
        out[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_frame_assignment_unit(ve):
    import ve_b200.dist as vd

    a = vd.frame_assignment(32, 0, 2, 64)
    b = vd.frame_assignment(32, 1, 2, 64)
    assert sorted(a + b) == list(range(64))
    assert vd.split_evenly(list(range(10)), 1, 3) == [3, 4, 5]


def test_gloo_world2_reductions():
    out = _run(2)
    assert set(out) == {0, 1}
    for r in (0, 1):
        rank, frames, t, n, err = out[r]
        assert frames != "error", t
        assert t == 2.0 and n == 300.0
        assert frames == [(r + 2 * i) % 64 for i in range(8)]


def test_gloo_failed_rank_is_an_error_not_a_hang():
    out = _run(2, fail_rank=1)
    rank, frames, t, n, err = out[0]
    assert frames != "error", t
    assert err is not None
