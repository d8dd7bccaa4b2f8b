"""The replica timing logic of bench.py with two ranks on CPU (gloo): every rank joins the process group,
the barrier returns on both, and dist_max gives every rank the largest of the ranks' times (the bench
reports the slowest replica's device time).  No GPU is touched."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, ws, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(ws),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    got_ws, got_rank, got_local = bench.dist_setup()
    bench.barrier(got_ws)
    m = bench.dist_max(1.5 + 10.0 * rank, got_ws)
    bench.barrier(got_ws)
    dist.destroy_process_group()
    q.put((rank, got_ws, got_rank, got_local, m))


def test_two_ranks_barrier_and_max():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[:4] for o in out] == [(0, 2, 0, 0), (1, 2, 1, 1)]
    assert all(o[4] == 11.5 for o in out)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.dist_max(3.25, 1) == 3.25
    bench.barrier(1)
