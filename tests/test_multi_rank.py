"""The multi-GPU harness of bench.py, on CPU with gloo (world size 2): one process per
rank, rendezvous on 127.0.0.1, max-over-ranks timing and barriers.  The product itself runs
as independent replicas (one per GPU); there is no collective on the data path."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, pg = bench.dist_setup(None)
    ms = bench.max_over_ranks(pg, 10.0 * (rank + 1))        # per-rank step time: the job takes the slowest
    bench.barrier(pg)
    q.put((r, w, local, ms))
    pg.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 2, 0, 20.0), (1, 2, 1, 20.0)]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    w, r, local, pg = bench.dist_setup(None)
    assert (w, r, local, pg) == (1, 0, 0, None)
    assert bench.max_over_ranks(pg, 3.5) == 3.5
