"""The multi-process path of bench.py on CPU (gloo, world size 2): replicas
on every rank, the step time taken as the maximum over ranks and the
whole-job value from it; the reference arm runs on rank 0 only."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        ms = bench.reduce_max(1.5 + rank, dist, "cpu")
        q.put((rank, ms, bench.replica_value(ws, ms)))
    finally:
        dist.destroy_process_group()


def test_replicas_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value in out:
        assert ms == 2.5  # the slower rank's time on every rank
        assert value == pytest.approx(2 * 1e3 / 2.5)  # evaluations of both ranks / max time


def _replica_rank(rank, ws, port, q):
    import time
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    log = []
    try:
        def timed_steps(k):
            # a replica whose steps take 1 + rank ms (rank 1 is the slow one)
            log.append(("steps", k, time.monotonic()))
            return [1.0 + rank] * k

        def barrier():
            dist.barrier()
            log.append(("barrier", 0, time.monotonic()))

        ms, value = bench.time_replicas(timed_steps, 3, 5, barrier,
                                        lambda v: bench.reduce_max(v, dist, "cpu"), ws)
        q.put((rank, ms, value, [e[:2] for e in log]))
    finally:
        dist.destroy_process_group()


def test_replica_timed_region_gloo():
    """The whole timed region of bench.py's replicas on two gloo ranks:
    warm-up, barrier, the timed steps, barrier, then the slowest rank's step
    time and the whole-job value, the same on every rank."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_replica_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value, log in out:
        assert log == [("steps", 3), ("barrier", 0), ("steps", 5), ("barrier", 0)]
        assert ms == 2.0  # rank 1's mean step
        assert value == pytest.approx(2 * 1e3 / 2.0)


def test_reference_arm_only_on_rank0():
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        steps, warmup = 1, 0

    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(Args(), 2, 1)
    assert buf.getvalue() == ""
