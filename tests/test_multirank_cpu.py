"""The multi-GPU bench path's host logic on two gloo ranks (CPU): every rank
builds its own shard of the workload (no data-path collective), and the
whole-job units are summed and the step times maxed over the ranks."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import importlib
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    bench = importlib.import_module("bench")
    rf = importlib.import_module("electron-integral-playground_b200.roofline")
    mols, pds, ads, stats = bench.build_workload(bench.shard_seed(0, rank), 2)
    tot, _ = rf.totals(stats)
    fake_ms = 10.0 + rank  # stands in for a rank's device time
    summed = bench.reduce_over_ranks([tot["screened"], tot["primitive"]], dist.ReduceOp.SUM, "cpu")
    slowest = bench.reduce_over_ranks([fake_ms], dist.ReduceOp.MAX, "cpu")[0]
    out.put((rank, [len(m.elements) for m in mols], tot["screened"], tot["primitive"], summed, slowest))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_and_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, atoms0, s0, p0, sum0, max0), (r1, atoms1, s1, p1, sum1, max1) = res
    assert atoms0 != atoms1 or s0 != s1  # independent shards
    assert sum0 == sum1 == [float(s0 + s1), float(p0 + p1)]
    assert max0 == max1 == 11.0


def test_single_process_reduction_is_identity():
    import importlib
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    bench = importlib.import_module("bench")
    assert bench.reduce_over_ranks([3, 4.5], None, "cpu") == [3.0, 4.5]
