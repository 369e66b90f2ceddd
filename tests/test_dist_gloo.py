"""The multi-process host logic with world_size 2 on CPU (gloo): the instance
partition is identical on every rank and balanced, timings combine as the
maximum over ranks, results gather back in instance order, and a rank that
fails surfaces as an error on the host rather than a hang."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from jaxiga_b200.dist import partition_by_cost


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_partition_is_deterministic_and_balanced():
    costs = [((i * 7919) % 97) ** 1.5 + 1 for i in range(256)]
    parts = partition_by_cost(costs, 4)
    assert sorted(i for p in parts for i in p) == list(range(256))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert parts == partition_by_cost(list(costs), 4)
    assert partition_by_cost([5.0], 3) == [[0], [], []]


def _worker(rank, world, port, q, fail_rank):
    import datetime

    import torch.distributed as dist

    from jaxiga_b200.dist import gather_by_index, max_over_ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        costs = [float(c) for c in [30, 10, 20, 5, 25, 15]]
        parts = partition_by_cost(costs, world)
        mine = parts[rank]
        t = max_over_ranks(1.0 + rank)
        if rank == fail_rank:
            raise RuntimeError("injected failure on the host")
        out = gather_by_index({i: i * i for i in mine}, parts, len(costs))
        q.put((rank, parts, t, out))
    except Exception as e:  # report, then leave the group
        q.put((rank, "error", repr(e), None))
    finally:
        dist.destroy_process_group()


def _run(world, fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    return sorted(res, key=lambda r: r[0])


def test_two_ranks_agree_on_partition_timing_and_results():
    res = _run(2)
    assert all(r[1] != "error" for r in res), res
    assert res[0][1] == res[1][1]
    assert res[0][2] == res[1][2] == 2.0
    assert res[0][3] == res[1][3] == [i * i for i in range(6)]


def test_a_failing_rank_is_reported_not_hung():
    res = _run(2, fail_rank=1)
    assert res[1][1] == "error" and "injected" in res[1][2]
    # the surviving rank's collective ends with an error or completes, within the timeout
    assert res[0][0] == 0
