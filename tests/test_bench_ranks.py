"""The multi-rank host logic of bench.py on CPU: two gloo ranks on
127.0.0.1 (one process per rank, as torchrun starts them on GPUs).  Each
rank solves its own replica (seed + rank), the job time is the max over
ranks, the reference arm prints from rank 0 only, and the batch workload's
fields are split across the ranks (disjoint, covering, balanced by cells)."""
import datetime
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sys.path.insert(0, ROOT)
        import bench
        t = bench.max_over_ranks(1.5 + rank, dist, "cpu")
        seed = bench.replica_seed(7, rank)

        class A:
            gpus, steps, warmup, cpu_sample_iters, nx, ny, seed = world, 1, 0, 1, 16, 8, 7
            batch_fields, batch_outer = 64, 200
        # the batch workload is split across the ranks: each rank's share,
        # gathered on every rank
        _, cells, mine = bench.batch_fields(A, rank, world)
        shares = [None] * world
        dist.all_gather_object(shares, (mine, [cells[q] for q in mine]))
        buf = io.StringIO()
        with redirect_stdout(buf):
            if rank != 0:
                bench.reference_arm(A, None, rank)     # must return without work or output
        dist.barrier()
        q.put((rank, t, seed, buf.getvalue(), shares))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=150) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.5, 2.5]            # max over ranks, seen by both
    assert [o[2] for o in out] == [7, 8]                # one replica per rank
    assert out[1][3] == ""                              # rank 1 of the reference arm prints nothing
    # batch fields: disjoint shares that cover all 64, of nearly equal work
    shares = out[0][4]
    assert shares == out[1][4]
    idx = [q for mine, _ in shares for q in mine]
    assert sorted(idx) == list(range(64))
    loads = [sum(c) for _, c in shares]
    assert abs(loads[0] - loads[1]) <= max(max(c) for _, c in shares)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, None, "cpu") == 3.25
    assert bench.replica_seed(0, 0) == 0
