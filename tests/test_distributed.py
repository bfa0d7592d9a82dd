"""The multi-process plumbing of bench.py (one rank per GPU, replicas) on
CPU: two gloo ranks run the barrier, the max-over-ranks timing and the
latency gather, and the ranks' problems are disjoint."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "CLAIRE_B200_DIST_BACKEND": "gloo"})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    r, w, _ = bench.dist_init()
    bench.barrier(w)
    mx = bench.max_over_ranks(10.0 * (r + 1), w)
    lats = bench.gather_list([100 * r + 1, 100 * r + 2], w)
    idx = bench.problem_indices(r, 4)
    all_idx = bench.gather_list(idx, w)
    dist.destroy_process_group()
    out.put((r, w, mx, lats, all_idx))


def test_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, mx, lats, all_idx in res:
        assert w == world
        assert mx == 20.0                          # max over ranks, on every rank
        assert lats == [1, 2, 101, 102]            # every rank's latencies, rank order
        assert sorted(all_idx) == list(range(8))   # disjoint problems, weak scaling
