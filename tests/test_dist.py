"""Multi-rank plumbing of bench.py on CPU: two gloo ranks, each a replica.

bench.py runs one process per GPU with no data-path collective; the ranks
only agree on the step time (maximum over ranks) and the total ray count
(sum over ranks). This checks those reductions with world size 2."""
import multiprocessing as mp
import os
import socket
import sys

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank(rank, world, port, queue):
    os.environ.update({'RANK': str(rank), 'LOCAL_RANK': str(rank), 'WORLD_SIZE': str(world),
                       'MASTER_ADDR': '127.0.0.1', 'MASTER_PORT': str(port), 'CUDA_VISIBLE_DEVICES': ''})
    sys.path.insert(0, str(ROOT))
    import bench
    dist = bench.Dist(world)
    try:
        dist.barrier()
        slowest = dist.max(10.0 + rank)
        total = dist.sum(100 * (rank + 1))
        queue.put((rank, slowest, total))
    finally:
        dist.close()


def test_two_gloo_ranks_reduce_time_and_rays():
    ctx = mp.get_context('spawn')
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results == [(0, 11.0, 300.0), (1, 11.0, 300.0)]
