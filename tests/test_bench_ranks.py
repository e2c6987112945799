"""Replica bookkeeping of bench.py with two gloo ranks on the CPU: the time reported is the slowest rank's, the rate
counts every rank's units, and the reference arm prints from rank 0 only."""
import contextlib
import io
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(1.0 + rank, "cpu")   # rank 1 is the slower one
        rate = bench.replica_rate(100, t, world)
        # the reference arm: rank 0 alone runs and prints (a stand-in potential: no reference library is needed)
        class FakeRef:
            def set_positions(self, frac):
                pass

            def eval(self):
                return None

        bench.reference_potential = lambda cores: (FakeRef(), 2724)

        class A:
            steps, warmup, gpus, pool, ref_seconds = 10, 3, world, 8, 0.05

        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            bench.run_reference(A())
        dist.barrier()
        out[rank] = (t, rate, buf.getvalue())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == pytest.approx(2.0) and res[1][0] == pytest.approx(2.0)
    assert res[0][1] == pytest.approx(100.0) and res[1][1] == pytest.approx(100.0)
    assert '"impl": "reference"' in res[0][2] and res[1][2] == ""
    import json
    line = json.loads(res[0][2])
    assert line["config"] == bench_config(2724, 8) and line["steps"] == 10 and line["e2e"]["value"] == line["value"]


def bench_config(M, P):
    sys.path.insert(0, ROOT)
    import bench
    return bench.workload_config(M, P)


def test_single_process_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert not dist.is_initialized()
    assert bench.max_over_ranks(3.5, "cpu") == 3.5
    assert bench.replica_rate(10, 2.0, 1) == 5.0
