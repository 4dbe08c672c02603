"""The N>1 path of bench.py on CPU ranks (gloo, world size 2): replicas
share nothing on the data path; the job is timed as its slowest rank and
counts every rank's frames; each rank searches its own seeded sequence."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    bench.barrier(world, device="cpu")
    slowest = bench.max_over_ranks(1.0 + rank, world, device="cpu")
    rate = bench.job_rate(world, 60, 3, slowest)
    from rivet_h26x_codecs_b200 import synth
    seq = synth.make_sequence(synth.HEVC, 64, 64, 8, 2, synth.seed_for(1, rank), 64, 64, 2.0)
    q.put((rank, slowest, rate, int(seq.frames[1].sum())))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_time_the_slowest_rank_and_count_every_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [2.0, 2.0]
    assert [o[2] for o in out] == [2 * 60 * 3 / 2.0] * 2
    assert out[0][3] != out[1][3], "ranks must search their own sequences"
