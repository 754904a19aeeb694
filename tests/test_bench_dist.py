"""The bench's multi-rank plumbing on CPU: two `gloo` ranks (one process each, as torchrun starts
them) meet at the barrier, agree on the max of their step times, and report the weak-scaling
aggregate (every rank's operations over the slowest rank's time)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), MAYO_BENCH_DIST_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    d.barrier()
    ms = 10.0 + 5.0 * rank  # this rank's step time
    ms_max = d.max(ms)
    d.barrier()
    out.put((rank, d.world, ms_max, bench.weak_value(1000.0, d.world, ms_max)))
    d.close()


def test_two_gloo_ranks_barrier_and_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    for _, world, ms_max, value in got:
        assert world == 2 and ms_max == pytest.approx(15.0)
        assert value == pytest.approx(1000.0 * 2 / 0.015)


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    assert d.world == 1 and d.pg is None
    assert d.max(3.5) == 3.5
    d.barrier()
