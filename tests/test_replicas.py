"""Replicas over a file list (CPU): the LPT partition, and the host-side
gather of per-rank results across two gloo processes, in list order."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from coherentsearch_c_b200.replicas import lpt_partition, search_list


def test_lpt_partition_covers_and_balances():
    rng = np.random.default_rng(1)
    costs = list(np.exp(rng.uniform(np.log(2e6), np.log(8e6), 256)))
    for n in (1, 2, 3, 8):
        parts = lpt_partition(costs, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT is within 4/3 of optimal; the optimum is at least the mean
        assert max(loads) <= (4.0 / 3.0) * max(sum(costs) / n, max(costs)) + 1e-6


def fake_search(idx):
    """Stands in for a GPU search: a deterministic per-file result."""
    return {i: np.arange(i % 7, dtype=np.float64) * (i + 1) for i in idx}


def _worker(rank, world, port, costs, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = search_list(costs, fake_search, dist)
        out_q.put((rank, [r.tolist() for r in res]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(120)
def test_two_ranks_gather_in_list_order():
    costs = [float(c) for c in np.random.default_rng(2).integers(1, 100, 23)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    want = [r.tolist() for r in search_list(costs, fake_search, None)]
    assert got[0] == want and got[1] == want


def failing_search(idx):
    """A rank whose search fails before the gather (the host-side stand-in
    for a replica that dies between steps)."""
    raise RuntimeError("replica failed")


def _worker_fault(rank, world, port, costs, out_q, mode):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    if mode == "never_joins" and rank == 1:
        out_q.put((rank, "absent"))
        return
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=5))
    except Exception as exc:   # noqa: BLE001
        out_q.put((rank, f"error: {type(exc).__name__}"))
        return
    try:
        fn = failing_search if (mode == "fails" and rank == 1) else fake_search
        search_list(costs, fn, dist)
        out_q.put((rank, "ok"))
    except Exception as exc:   # noqa: BLE001
        out_q.put((rank, f"error: {type(exc).__name__}"))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
@pytest.mark.parametrize("mode", ["fails", "never_joins"])
def test_a_lost_rank_ends_the_others_with_an_error(mode):
    """A rank that fails before the gather, or never joins, makes the other
    rank's collective (or rendezvous) end with an error within the process
    group's short timeout instead of waiting for good."""
    costs = [float(c) for c in range(1, 12)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_fault, args=(r, 2, port, costs, q, mode))
             for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert not p.is_alive()
    assert got[0].startswith("error")
    assert got[1] == ("absent" if mode == "never_joins" else "error: RuntimeError")
