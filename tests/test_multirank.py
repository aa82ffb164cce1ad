"""Multi-GPU host logic on the CPU: two ranks over gloo (127.0.0.1).

Frames are independent, so each rank scores its own frames (weak scaling)
and the only exchange is the max over ranks of the step timings.  This runs
the bench's own helpers for that in two processes: both ranks must agree on
the slowest rank's time, draw different frames, and count every rank's pixels
in the whole-job value."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, REPO)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        # rank r measured (10 + r) ms for the step and (3 - r) ms for the kernel
        got = bench.max_over_ranks(dist, [10.0 + rank, 3.0 - rank], "cpu")
        seeds = [bench.rank_seed(0x5EED1000, rank) + f for f in range(64)]
        value = bench.whole_job_mpix(world, 64 * 1024 * 1024, got[0])
        out.put((rank, got, seeds[0], seeds[-1], value))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_ranks_share_the_slowest_time_and_score_different_frames():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=100) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    results.sort()
    for _, got, _, _, value in results:
        assert got == [11.0, 3.0]  # the slowest rank's step, the slowest kernel
        assert value == pytest.approx(2 * 64 * 1024 * 1024 / 0.011 / 1e6)
    # the ranks' frame seeds do not overlap
    (_, _, a0, a1, _), (_, _, b0, b1, _) = results
    assert a1 < b0 or b1 < a0
