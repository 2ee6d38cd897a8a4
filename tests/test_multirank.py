"""The multi-rank host logic of bench.py on CPU: two gloo ranks (world size 2, 127.0.0.1).
`--gpus N` runs N independent replicas of the step (the torus update on one grid is not
sharded, so no data-path collective exists); what the ranks share is the barrier around the
timed region and the maximum of their times.  Checked here: max_over_ranks returns the
largest rank value on every rank, the barriers pair up, and the reference arm does its work
on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(ws),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import io
    import contextlib
    import bench
    import torch.distributed as dist

    class A:
        impl = "reference"
    w, r, _ = bench.dist_init(A())
    assert (w, r) == (ws, rank)
    bench.barrier(ws)
    got = bench.max_over_ranks(1.5 + 2.0 * rank, ws)
    bench.barrier(ws)
    # the reference arm: rank 0 alone runs and prints; the others return without work
    printed = ""
    if rank != 0:
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            bench.run_reference(None, ws, rank)
        printed = buf.getvalue()
    out.put((rank, got, printed))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_share_max_and_barrier():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = {}
    try:
        for _ in range(ws):
            rank, got, printed = q.get(timeout=120)
            res[rank] = (got, printed)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert res[0][0] == res[1][0] == pytest.approx(3.5)
    assert res[1][1] == ""
