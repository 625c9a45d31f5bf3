"""The multi-GPU form of the benchmark is replicas only (independent coarse channels per
rank, no collective on the data path): its host logic -- per-rank seeds, the max-over-ranks
time and the whole-job throughput -- checked with two gloo ranks on the CPU, and the
reference arm's rank behaviour."""
import contextlib
import io
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    local_ms = [3.0, 5.0][rank]  # rank 1 is the slow replica
    t_max = bench.max_over_ranks(local_ms, world)
    value = bench.replica_value(100, 4, world, t_max * 1e-3)
    dist.barrier()
    out.put((rank, t_max, value, bench.rank_seeds(rank, 4)))
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, v0, s0), (r1, t1, v1, s1) = res
    assert t0 == t1 == 5.0                       # every rank reports the slowest replica
    assert v0 == v1 == 100 * 4 * 2 / 5e-3        # all ranks' units over that time
    assert not set(s0) & set(s1)                 # independent channels per rank


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(2.5, 1) == 2.5
    assert bench.replica_value(10, 2, 1, 0.5) == 40.0


def test_reference_arm_runs_on_rank_zero_only():
    class A:
        steps, warmup = 1, 0
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        assert bench.run_reference(A, 1, 2) == 0
    assert buf.getvalue() == ""
