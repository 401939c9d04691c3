"""The multi-rank plumbing of bench.py on CPU: two `gloo` ranks (127.0.0.1), as `torchrun --nproc-per-node 2`
would start them.  The path shards into independent replicas (no collective on the data path); what
the ranks share is the timing: every rank contributes its total time, the job's time is the slowest
rank's (max over ranks), and the job's rate counts every rank's work."""
import contextlib
import io
import os
import socket
import sys
from datetime import timedelta
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    t = bench._max_over_ranks(100.0 + 50.0 * rank, world, device="cpu")   # rank 1 is the slower one
    rate = bench.replica_rate(1_000_000, world, 4, t)
    # the reference arm: every rank but rank 0 leaves without work or output
    buf = io.StringIO()
    if rank != 0:
        with contextlib.redirect_stdout(buf):
            bench.run_reference_arm(None, rank, world)
    dist.barrier()
    q.put((rank, t, rate, buf.getvalue()))
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, rate, out in got:
        assert t == 150.0                          # max over ranks
        assert rate == pytest.approx(2 * 4 * 1_000_000 / 0.150 / 1e6)
        assert out == ""
