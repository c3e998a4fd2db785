"""Multi-rank host logic of bench.py on CPU: world size 2 over gloo.

The solve itself runs as independent replicas (one per GPU, no data-path
collective), so what spans ranks is the benchmark's host logic: the barrier
around the timed region, the max over ranks of the measured time, rank 0
alone printing, the reference arm's rank-0-only run, and a departed rank
ending the others' next collective with an error instead of a hang.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_env(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)


def _max_worker(rank, world, port, q):
    _rank_env(rank, world, port)
    import bench
    w, r, _, pg = bench.dist_setup(None, backend="gloo", timeout_s=30)
    bench.barrier(pg)
    q.put((r, w, bench.max_over_ranks(pg, 1.5 + r)))
    bench.barrier(pg)
    pg.destroy_process_group()


def _leave_worker(rank, world, port, q):
    _rank_env(rank, world, port)
    import bench
    _, r, _, pg = bench.dist_setup(None, backend="gloo", timeout_s=5)
    bench.barrier(pg)
    if r == 1:
        q.put((r, "left"))
        q.close()
        q.join_thread()   # the message is out before the process goes
        os._exit(0)       # leaves between steps, with nothing in flight
    try:
        bench.barrier(pg)
        q.put((r, "no error"))
    except Exception as e:   # gloo: peer closed, or the timeout
        q.put((r, "error: %s" % type(e).__name__))


def _run(target, world=2, timeout=90):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = []
    try:
        for _ in range(world):
            out.append(q.get(timeout=timeout))
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    return sorted(out)


def test_max_over_ranks_and_barrier_gloo():
    out = _run(_max_worker)
    assert [o[0] for o in out] == [0, 1]
    for _, world, v in out:
        assert world == 2
        assert v == 2.5   # the slowest rank's value on every rank


def test_departed_rank_ends_next_collective_with_error():
    out = dict(_run(_leave_worker))
    assert out[1] == "left"
    assert out[0].startswith("error"), out[0]


def test_reference_arm_rank0_only_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
