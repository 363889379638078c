"""The multi-rank logic of bench.py on CPU: two gloo ranks, each timing its own
replica, reduce to the slowest rank's time, and the whole-job rate counts every
rank's steps.  (One process per GPU under torchrun on a GPU node; here the same
host code runs with the gloo backend.)"""
import importlib.util
import os
import socket
from datetime import timedelta

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    b = _bench()
    ms = b.max_over_ranks(100.0 + 7.0 * rank, dist, "cpu")  # rank r took 100 + 7r ms for its steps
    q.put((rank, ms, b.whole_job_rate(world, 50, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_to_the_slowest_rank():
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
    assert [o[1] for o in out] == [107.0, 107.0]
    assert all(abs(o[2] - 2 * 50 / 0.107) < 1e-9 for o in out)


def test_single_process_needs_no_group():
    b = _bench()
    assert b.max_over_ranks(3.5, None, "cpu") == 3.5
    assert b.whole_job_rate(1, 10, 20.0) == 500.0
