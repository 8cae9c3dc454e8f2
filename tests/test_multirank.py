"""Multi-process plumbing of bench.py on CPU (gloo, world size 2).

The path runs as independent replicas, one per GPU, with no collective on
the data path: the only cross-rank step is the maximum of the per-rank
timings, from which rank 0 forms the whole-job rate.  Here two gloo ranks
report different timings and must agree on the maximum; a rank that never
joins makes the other's collective fail within the process-group timeout
instead of hanging.
"""
import datetime
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, timings, out_q, skip_rank):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    if rank == skip_rank:
        return  # this rank never joins
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
        dev, wall = bench.max_over_ranks(timings[rank], dist, "cpu")
        value, e2e = bench.replica_rates(100, world, dev, wall)
        out_q.put((rank, dev, wall, value, e2e))
    except Exception as e:  # noqa: BLE001
        out_q.put((rank, "error", type(e).__name__))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def run(world, timings, skip_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, timings, q, skip_rank)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(60)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive
    out = []
    while not q.empty():
        out.append(q.get())
    return sorted(out)


def test_replica_timing_is_the_max_over_ranks():
    timings = [[0.50, 0.80], [0.65, 0.70]]
    out = run(2, timings)
    assert len(out) == 2
    for rank, dev, wall, value, e2e in out:
        assert dev == 0.65 and wall == 0.80
        assert value == pytest.approx(200 / 0.65) and e2e == pytest.approx(200 / 0.80)


def test_missing_rank_fails_instead_of_hanging():
    out = run(2, [[1.0, 1.0], [1.0, 1.0]], skip_rank=1)
    # rank 0 either cannot rendezvous or its collective times out: an error, not a hang
    assert len(out) == 1 and out[0][0] == 0 and out[0][1] == "error", out
