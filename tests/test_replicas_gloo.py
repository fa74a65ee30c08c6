"""The benchmark's multi-rank bookkeeping (replicas, no data-path collective) with
world_size 2 over gloo on CPU: max-over-ranks timing, the whole-job throughput,
and the reference arm's non-zero ranks exiting without work."""

import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import types

    import torch.distributed as dist

    import bench
    w, r, _ = bench.init_dist("gloo")
    ms_local = 100.0 + 50.0 * r  # rank 1 is the slow one
    value, ms = bench.job_throughput(ms_local, w, 10)
    bench.barrier(w)
    args = types.SimpleNamespace(steps=1, warmup=0)
    ref_rc = bench.run_reference(args) if r != 0 else None
    dist.destroy_process_group()
    q.put((r, w, value, ms, ref_rc))


def test_replicas_max_over_ranks_gloo():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for r, w, value, ms, ref_rc in out:
        assert w == 2 and ms == 150.0  # the slowest rank's time on every rank
        assert abs(value - 2 * 10 / 0.150) < 1e-9
        if r != 0:
            assert ref_rc == 0  # the reference arm runs on rank 0 only
