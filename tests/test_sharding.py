"""Block partition and ghost-cell halo exchange across two ranks (gloo on CPU).

Each rank owns contiguous Morton ranges of blocks on every AMR level
(sharding.partition).  Starting from a field whose blocks are all set on
rank 0's view but whose non-owned blocks are NaN on each rank, every pass of
the three-pass ghost fill (AMR level ascending, x then y then z;
fmg_ghostcell.F90:43-55) is preceded by that pass's exchange
(GhostExchange.pass_exchange) and then computed by the oracle's pass on the
rank's field.  A rank's owned blocks must then hold, bit for bit, what one
rank computes for the whole hierarchy -- no value read from a block another
rank owns may be missing or stale, or a NaN (or a wrong value) appears.
Hierarchies: periodic with 3 AMR levels (same-level and coarse-fine faces),
isolated with physical-boundary faces; fmg levels n = 8 and n = 2, bilinear
and bicubic coarse-fine ghosts.
"""
import os
import socket
import time

import numpy as np
import pytest
import torch.multiprocessing as mp

CASES = [("periodic", 0, False), ("periodic", 2, False), ("periodic", 0, True), ("sphere", 0, True),
         ("sphere", 1, False)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _hier(kind):
    from code_only_b200 import workloads as w
    return w.small_periodic(2, 8, 3, 1) if kind == "periodic" else w.small_sphere(2, 8, 3, 2)


def _field(h, f):
    n = h.ni >> f
    G = n + 2
    return np.random.default_rng(123 + f).standard_normal((h.nblocks, G, G, G))


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist
    from code_only_b200 import sharding
    from tests.oracle_lib import oracle_ghost_pass
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        for kind, f, cubic in CASES:
            h = _hier(kind)
            n = h.ni >> f
            owner = sharding.partition(h, world)
            ex = sharding.GhostExchange(h, owner, rank, n)
            a = _field(h, f)
            a[owner != rank] = np.nan          # another rank's blocks are unknown here
            t = torch.from_numpy(a.reshape(-1))   # shares memory with a
            for L in range(h.nlev):
                for d in range(3):
                    ex.pass_exchange(t, L, d)
                    oracle_ghost_pass(h, a, f, L, d, cubic)
            mine = owner == rank
            q.put((rank, kind, f, cubic, a[mine].copy(), int(mine.sum()),
                   sum(ex.bytes_per_pass().values())))
        q.put((rank, "max", sharding.allreduce_max(float(rank + 1))))
    finally:
        dist.destroy_process_group()


def _run(world=2, timeout=240):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = []
    t0 = time.time()
    while len(out) < world * (len(CASES) + 1) and time.time() - t0 < timeout:
        try:
            out.append(q.get(timeout=5))
        except Exception:
            if not any(p.is_alive() for p in procs):
                break
    for p in procs:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    return out


@pytest.fixture(scope="module")
def two_ranks():
    return _run()


def test_partition_is_balanced_and_contiguous():
    from code_only_b200 import sharding
    h = _hier("periodic")
    for world in (1, 2, 3, 4):
        owner = sharding.partition(h, world)
        for L in range(h.nlev):
            o = owner[h.level == L]
            assert np.all(np.diff(o) >= 0)                       # contiguous ranges in Morton order
            counts = np.bincount(o, minlength=world)
            assert counts.max() - counts.min() <= 1


@pytest.mark.parametrize("case", CASES, ids=[f"{k}-f{f}-{'cubic' if c else 'linear'}" for k, f, c in CASES])
def test_two_rank_ghost_fill_is_bitwise(two_ranks, case):
    from code_only_b200 import sharding
    from tests.oracle_lib import oracle_ghost_pass
    kind, f, cubic = case
    h = _hier(kind)
    ref = _field(h, f)
    oracle_ghost_pass(h, ref, f, -1, 0, cubic)         # the whole fill on one rank
    owner = sharding.partition(h, 2)
    got = {r: v for (r, k, ff, c, v, cnt, nbytes) in
           [x for x in two_ranks if x[1] != "max"] if (k, ff, c) == case}
    assert set(got) == {0, 1}, "a rank did not report"
    for r in (0, 1):
        assert np.isfinite(got[r]).all()
        assert np.array_equal(got[r], ref[owner == r])


def test_allreduce_max(two_ranks):
    vals = [x[2] for x in two_ranks if x[1] == "max"]
    assert vals == [2.0, 2.0]
