"""The N > 1 plumbing on CPU: two gloo ranks (spawned processes) agree on
the max / sum reductions the benchmark uses and on the placement rank 0
broadcasts; least_loaded places sessions by free budget."""
import os
import socket

import pytest

from dynamap_b200.replicas import Ranks, least_loaded


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    r = Ranks(backend="gloo", timeout_s=60)
    try:
        r.barrier()
        t = 1.5 + rank           # per-rank device time
        frames = 100 * (rank + 1)
        place = r.broadcast(least_loaded([5, 4, 3], [8, 8])[0] if rank == 0 else None)
        out.put((rank, r.max(t), r.sum(frames), place))
    finally:
        r.close()


def test_two_gloo_ranks_agree():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    for _, tmax, fsum, place in got:
        assert tmax == pytest.approx(2.5)      # the slower rank bounds the job
        assert fsum == pytest.approx(300.0)    # frames of both ranks
        assert place == [0, 1, 1]              # rank 0's decision on both ranks


def test_single_process_is_identity():
    r = Ranks()
    assert (r.world, r.rank) == (1, 0)
    assert r.max(3.0) == 3.0 and r.sum(2.0) == 2.0 and r.broadcast("x") == "x"
    r.close()


def test_least_loaded_placement():
    place, free = least_loaded([6, 6, 6, 10], [12, 10])
    assert place == [0, 1, 0, -1]
    assert free == [0, 4]
    place, _ = least_loaded([1, 1, 1], [5, 5, 5])
    assert place == [0, 1, 2]
