"""Host logic of the N-GPU runs, on CPU with two gloo ranks: the max / sum
over ranks that bench.py reports (the time of a run is the slowest rank's),
the work-balanced split of a batch's instances, gathering per-rank latency
lists, and a rank that fails before a collective turning into an error on
the other rank rather than a hang."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from fvstuff_b200 import ranks as R  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    try:
        dist = R.init("gloo", timeout_s=20)
        if mode == "fail" and rank == 1:
            raise SystemExit(3)  # leaves before the collective
        # a run's time is the slowest rank's; work and counters add up
        t = R.max_over_ranks(1.0 + rank, dist)
        w = R.sum_over_ranks(10.0 * (rank + 1), dist)
        lat = R.gather([rank, rank + 0.5], dist)
        costs = [float(n) ** 3 for n in (64, 512, 96, 480, 128, 448, 160, 416, 192, 384)]
        mine = R.shard_by_work(costs, rank, world)
        parts = R.gather(mine, dist)
        R.finish(dist)
        q.put((rank, "ok", t, w, lat, parts))
    except SystemExit:
        raise
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e)))


def _spawn(mode, world=2):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank hung"
    out = {}
    while not q.empty():
        item = q.get()
        out[item[0]] = item[1:]
    return procs, out


def test_two_ranks_reduce_gather_and_split():
    procs, out = _spawn("ok")
    assert all(p.exitcode == 0 for p in procs)
    costs = [float(n) ** 3 for n in (64, 512, 96, 480, 128, 448, 160, 416, 192, 384)]
    for rank in (0, 1):
        status, t, w, lat, parts = out[rank]
        assert status == "ok"
        assert t == 2.0 and w == 30.0
        assert lat == [[0, 0.5], [1, 1.5]]
        # both ranks computed the same partition: disjoint and complete
        assert sorted(parts[0] + parts[1]) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - sum(costs) / 2 <= max(costs)


def test_rank_leaving_before_a_collective_is_an_error_not_a_hang():
    procs, out = _spawn("fail")
    assert procs[1].exitcode == 3
    assert out[0][0] == "error"


def test_split_single_process_and_balance():
    costs = [5.0, 1.0, 4.0, 2.0, 3.0]
    assert R.shard_by_work(costs, 0, 1) == [0, 1, 2, 3, 4]
    parts = [R.shard_by_work(costs, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == [0, 1, 2, 3, 4]
    assert [sum(costs[i] for i in p) for p in parts] == [5.0, 5.0, 5.0]
    assert R.max_over_ranks(2.5) == 2.5 and R.sum_over_ranks(4.0) == 4.0 and R.gather("x") == ["x"]


@pytest.mark.parametrize("world", [2, 4])
def test_split_is_deterministic(world):
    costs = [float((k * 37) % 17 + 1) for k in range(40)]
    parts = [R.shard_by_work(costs, r, world) for r in range(world)]
    assert parts == [R.shard_by_work(costs, r, world) for r in range(world)]
    assert sorted(sum(parts, [])) == list(range(40))
