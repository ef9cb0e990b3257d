"""Multi-rank plumbing of bench.py, exercised with two gloo ranks on the CPU.

The fit-null path does not shard (each GPU fits its own cohort), so the only
cross-rank steps are the barrier and the max-over-ranks reduction of the
device-timed step; the reference arm runs on rank 0 alone.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_q) -> None:
    sys.path.insert(0, str(ROOT))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        step_max = bench.reduce_max(1.5 + rank, world, "cpu")
        out_q.put((rank, step_max, bench.whole_job_seconds_per_fit(step_max, world)))
    finally:
        dist.destroy_process_group()


def test_step_time_is_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [2.5, 2.5]      # both ranks see the slowest rank's time
    assert [g[2] for g in got] == [1.25, 1.25]    # two fits completed in 2.5 s


def test_single_rank_reduction_is_identity():
    import bench

    assert bench.reduce_max(3.25, 1, "cpu") == 3.25
    assert bench.whole_job_seconds_per_fit(3.25, 1) == 3.25


def test_reference_arm_runs_on_rank_zero_only():
    import bench

    saved = sys.argv
    sys.argv = ["bench.py", "--impl", "reference"]
    try:
        args = bench.parse_args()
    finally:
        sys.argv = saved
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args, rank=1)
    assert buf.getvalue() == ""
