"""The multi-GPU form of the benchmark is replicas only: each rank solves its own frequencies and the timing is the
max over ranks. Its host logic with world_size 2 over gloo on the CPU (no GPU, no data-path collective)."""
import os
import socket

import pytest

torch = pytest.importorskip('torch')
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = bench.rank_frequencies(rank, world)
        t = bench.max_over_ranks([1.0 + rank, 10.0 - rank], world, 'cpu')
        out.put((rank, mine, t))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_the_sweep_and_take_the_max_time():
    import bench
    world = 2
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    (r0, f0, t0), (r1, f1, t1) = res
    assert not set(f0) & set(f1)                                         # no frequency solved twice
    assert sorted(f0 + f1) == sorted(float(f) for f in bench.FREQS)      # the whole sweep
    assert t0 == t1 == [2.0, 10.0]                                       # the max over ranks, on every rank
    assert bench.rank_frequencies(0, 1)[:3] == [float(bench.FREQS[i]) for i in (0, 8, 16)]
