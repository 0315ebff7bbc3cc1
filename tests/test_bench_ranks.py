"""The multi-rank host logic of bench.py on the CPU: two gloo ranks (no GPU)
agree on the max-over-ranks time, the whole-job rate counts every replica,
and the reference arm runs on rank 0 only."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

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
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + rank, device="cpu")
        out.put((rank, ms, bench.replica_rate(world, 1000, 4, 5, ms)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    import torch.multiprocessing as mp
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
    assert [r[1] for r in res] == [11.0, 11.0]
    assert res[0][2] == res[1][2] == pytest.approx(2 * 1000 * 4 * 5 / 11e-3)


def test_max_over_ranks_without_a_process_group_is_the_rank_value():
    assert bench.max_over_ranks(3.5, device="cpu") == 3.5


def test_reference_arm_prints_nothing_off_rank_zero():
    class A:
        steps, warmup = 1, 3
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(A(), rank=1, world=2)
    assert buf.getvalue() == ""


def test_reference_arm_line_or_unavailable_on_rank_zero():
    """Rank 0 prints one JSON line: the reference's numbers, or `unavailable`."""
    import oracle
    if oracle.reference() is not None:
        pytest.skip("the reference is built here: the full arm runs for minutes")

    class A:
        steps, warmup = 1, 3
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(A(), rank=0, world=1)
    d = json.loads(buf.getvalue())
    assert d["impl"] == "reference" and "unavailable" in d
