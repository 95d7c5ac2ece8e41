"""The N > 1 path of bench.py (independent replicas): two gloo ranks on CPU agree on the
slowest rank's time and the whole-job value; the reference arm runs on rank 0 only."""
import importlib.util
import os
import socket
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    b = _bench()
    w, r, local, dist = b.dist_setup()
    try:
        t = b.reduce_max(dist, 1.0 + r)          # rank 1 is the slower replica
        out[r] = (w, t, b.aggregate_value(w, 3, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == out[1] == (2, 2.0, 3.0)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    b = _bench()

    class A:
        pass
    assert b.run_reference(A(), 2, 1) is None     # rank 1 exits without work
    assert capsys.readouterr().out == ""
