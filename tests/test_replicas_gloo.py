"""The bench's multi-GPU form (replicas, one process per GPU) on the CPU:
two ranks over gloo run its rank setup, its max / sum reductions of the
timed values, its barrier, and its split of the workloads' graph indices.
Replicas solve independent graphs, so the only exchange is these scalar
reductions; no data-path collective exists to test."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    w, r, local, pg = bench.dist_setup()
    mx = bench.max_over_ranks(pg, float(r + 1) * 10.0)
    total = bench.sum_over_ranks(pg, 4096.0)
    bench.barrier(pg)
    ranges = bench.rank_index_ranges(r, mix_graphs=4096, tune_graphs=128, serve_requests=20000, calib_graphs=512)
    q.put((r, w, local, mx, total, ranges))
    pg.destroy_process_group()


def test_two_replicas_over_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(2):
            r, w, local, mx, total, ranges = q.get(timeout=120)
            got[r] = (w, local, mx, total, ranges)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert sorted(got) == [0, 1]
    for r, (w, local, mx, total, _) in got.items():
        assert (w, local) == (2, r)
        assert mx == 20.0          # the slower replica's time
        assert total == 8192.0     # the work of both replicas
    spans = [span for r in got for span in got[r][4].values()]
    spans.sort()
    for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
        assert a1 <= b0, (spans,)  # no graph index is used twice
