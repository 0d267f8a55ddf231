"""The multi-GPU plumbing of bench.py on CPU: world size 2 over gloo.  The
path has no exchange step (independent replicas, one process per GPU), so
what is shared is the barrier around the timed region, the max over ranks of
its duration, and rank 0 alone printing -- or alone running the reference
arm."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import io
    import contextlib
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_init("gloo")
    try:
        bench.barrier(w)
        longest = bench.max_over_ranks(10.0 * (r + 1), w)
        # the reference arm: every rank but 0 returns at once, printing nothing
        out = io.StringIO()
        ran = None
        if r != 0:
            class A:
                steps, warmup = 1, 0
            with contextlib.redirect_stdout(out):
                for fn in (bench.run_reference, bench.run_reference_sk, bench.run_reference_ifb,
                           bench.run_reference_c3, bench.run_reference_c5):
                    fn(A(), {}, w, r)
            ran = out.getvalue()
        bench.barrier(w)
        q.put((r, w, longest, ran))
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, *_ in res] == [0, 1]
    assert all(w == 2 for _, w, _, _ in res)
    # the timed duration every rank reports is the slowest rank's
    assert all(longest == 20.0 for _, _, longest, _ in res)
    # rank 1's reference arm did nothing and printed nothing
    assert res[1][3] == ""
