"""The multi-rank plumbing of bench.py on CPU: two gloo ranks started the
way torchrun starts them (RANK / WORLD_SIZE / MASTER_* in the environment),
each timing its own replica.  The timing reduction is the maximum over the
ranks, the whole-job value counts every rank's replica, and the reference
arm runs on rank 0 only."""
import importlib.util
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    b = _bench()
    r, w, local, dist = b.dist_setup(world, backend="gloo")
    try:
        # rank r "took" 1 + r seconds for its replica of 0.05 simulated ps
        t = b.max_over_ranks(dist, 1.0 + r, "cpu")
        out[r] = (r, w, t, b.replica_throughput(w, 0.05, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_timing_to_the_slowest():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(out.keys()) == [0, 1]
    for r in range(2):
        rank, world, t, value = out[r]
        assert world == 2 and t == 2.0  # the slowest rank's time on every rank
        assert value == pytest.approx(2 * 0.05 / (2.0 / 3600.0))


def _ref_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world))
    b = _bench()
    calls = []

    class Args:
        config = "c1"
        steps = 1
        warmup = 0

    b.load_pkg = lambda: calls.append("work") or (_ for _ in ()).throw(RuntimeError("rank 0 only"))
    try:
        b.reference_arm(Args())
        out[rank] = "returned"
    except RuntimeError:
        out[rank] = "worked"


def test_reference_arm_runs_on_rank_zero_only():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_ref_main, args=(r, 2, 0, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert out[0] == "worked"      # rank 0 starts the oracle work
    assert out[1] == "returned"    # the other ranks exit without work
