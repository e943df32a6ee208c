"""Multi-rank replica driver on CPU (gloo, world size 2): throughput is all
ranks' solves over the slowest rank's time, and a failing rank ends the
others' collectives with an error instead of a hang."""
import os
import socket
import time

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from code_only_b200 import replicas
    info = replicas.setup("gloo", timeout_s=20.0)
    try:
        if mode == "timing":
            delay = 0.01 * (rank + 1)       # rank 1 is the slow one
            step = lambda: time.sleep(delay)

            def clock(fn, k):
                t = time.perf_counter()
                for _ in range(k):
                    fn()
                return (time.perf_counter() - t) * 1e3

            r = replicas.timed_replicas(info, step, steps=5, warmup=1, clock=clock)
            q.put((rank, r))
        else:
            if rank == 1:
                raise RuntimeError("injected failure on rank 1")
            try:
                replicas.max_over_ranks(info, 1.0)
                q.put((rank, "no error"))
            except Exception as e:          # the peer vanished: the collective fails
                q.put((rank, "error: " + type(e).__name__))
    finally:
        if mode == "timing":
            replicas.teardown(info)


def _run(mode, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    t0 = time.time()
    while len(out) < (2 if mode == "timing" else 1) and time.time() - t0 < timeout:
        try:
            r, v = q.get(timeout=5)
            out[r] = v
        except Exception:
            pass
    for p in procs:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    return out


def test_weak_scaling_throughput_uses_slowest_rank():
    out = _run("timing")
    assert set(out) == {0, 1}
    for r in (0, 1):
        res = out[r]
        assert res["world"] == 2
        # slowest rank: 5 x 20 ms; 10 solves over ~100 ms
        assert 18.0 <= res["ms_per_step"] <= 60.0
        assert abs(res["solves_per_s"] - 2 * 1e3 / res["ms_per_step"]) < 1e-6 * res["solves_per_s"]


def test_failing_rank_does_not_hang_the_others():
    out = _run("failure", timeout=90)
    assert out.get(0, "").startswith("error"), out
