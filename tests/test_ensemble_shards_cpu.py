"""Sharding one seeded ensemble over ranks (the multi-GPU form of the ensemble
workload: independent cases, no data-path collective) and gathering every case's
forces: a deterministic cost-balanced partition, checked for coverage,
disjointness and balance, and a two-rank gloo gather of fake per-case forces."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest


def test_partition_covers_every_case_once_and_balances_cost(ib):
    probs = ib.configs.ensemble_cases(128, seed=2026)
    costs = [ib.ensemble.case_cost(p) for p in probs]
    for world in (1, 2, 3, 4, 8):
        parts = ib.ensemble.shard_cases(costs, world)
        assert len(parts) == world
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(costs)))  # disjoint and covering
        loads = [sum(costs[k] for k in p) for p in parts]
        # greedy by decreasing cost: no rank exceeds the mean by more than one case
        assert max(loads) - sum(loads) / world <= max(costs)
        assert max(loads) <= 1.05 * sum(loads) / world or world == 1
        assert parts == ib.ensemble.shard_cases(costs, world)  # same on every rank


def test_partition_rejects_zero_ranks(ib):
    with pytest.raises(ValueError):
        ib.ensemble.shard_cases([1, 2], 0)


def _worker(rank, world, port, q):
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import __graft_entry__ as ge

    ib = ge.load_package()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    costs = [(k % 3 + 1) * 1000 for k in range(11)]
    mine = ib.ensemble.shard_cases(costs, world)[rank]
    fake = np.array([[k + 0.25, -k - 0.5] for k in mine])  # the forces case k would report
    table = ib.ensemble.gather_case_forces(len(costs), mine, fake, dist, "cpu")
    # a rank that claims a case another rank owns is caught
    dup = mine + ([0] if 0 not in mine else [])
    err = None
    try:
        ib.ensemble.gather_case_forces(len(costs), dup, np.zeros((len(dup), 2)), dist, "cpu")
    except ValueError as e:
        err = str(e)
    q.put((rank, mine, table.tolist(), err))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_gather_every_case():
    import torch.multiprocessing as mp

    with socket.socket() as sck:
        sck.bind(("127.0.0.1", 0))
        port = sck.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owned = sorted(out[0][1] + out[1][1])
    assert owned == list(range(11)) and not set(out[0][1]) & set(out[1][1])
    expect = [[k + 0.25, -k - 0.5] for k in range(11)]
    assert out[0][2] == expect and out[1][2] == expect
    assert out[0][3] is not None and "exactly one" in out[0][3]
