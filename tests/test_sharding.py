"""Block partition and halo exchange across two ranks (gloo on CPU).

Each rank owns contiguous Morton ranges of blocks on every AMR level
(sharding.partition) and holds NaN in the blocks it does not own.

Ghost fill: every pass of the three-pass fill (AMR level ascending, x then
y then z; fmg_ghostcell.F90:43-55) is preceded by that pass's exchange
(HaloExchange.ghost) and then computed by the oracle's pass on the rank's
field.

Composite operator: red-black sweeps (fmg_poisson_relax) and residuals
(fmg_poisson_resid) run as the oracle's pieces restricted to the rank's own
blocks (oracle_step), with the converge, ghost-pass and flux-correction
exchanges before the pieces that read other blocks, and the residual maximum
all-reduced.

AMR-level V-cycle: the prolongation onto every level (parent blocks to the
children's owners) and the base-grid solve (every base block to every
rank), likewise.

The whole solve: the oracle's fmg_cycle on each rank's blocks
(oracle_solve_split), which calls back before every step that reads
another rank's blocks, for every maximum and every ordered sum.

Owners are contiguous Morton ranges per level (sharding.partition) and,
to put most neighbours, parents and children on the other rank, alternating
blocks; with alternating owners, turning any one kind of exchange into a
no-op must leave NaN in the owned blocks.

A rank's owned blocks must then hold, bit for bit, what one rank computes
for the whole hierarchy -- no value read from a block another rank owns may
be missing or stale, or a NaN (or a wrong value) appears.  Hierarchies:
periodic with 3 AMR levels (same-level and coarse-fine faces), isolated
with physical-boundary faces; fmg levels n = 8, 4 and 2, bilinear and
bicubic coarse-fine ghosts.
"""
import os
import socket
import time

import numpy as np
import pytest
import torch.multiprocessing as mp

CASES = [("periodic", 0, False), ("periodic", 2, False), ("periodic", 0, True), ("sphere", 0, True),
         ("sphere", 1, False)]
# composite-operator cases: (hierarchy, fmg level)
OP_CASES = [("periodic", 0), ("periodic", 1), ("periodic", 2), ("sphere", 0)]
SWEEPS = 2
# AMR-level V-cycle transfers (prolongation, base-grid solve) at the vmg
# blocks' fmg level
VMG_CASES = ["periodic", "sphere"]
# owners: contiguous Morton ranges per level (sharding.partition), and
# alternating blocks, which puts most neighbours, parents and children of a
# block on the other rank
PARTS = ["morton", "alternating"]


def _owner(h, part, world=2):
    from code_only_b200 import sharding
    if part == "morton":
        return sharding.partition(h, world)
    if part == "nested":
        return sharding.partition(h, world, nested=True)
    return (np.arange(h.nblocks) % world).astype(np.int32)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _hier(kind):
    from code_only_b200 import workloads as w
    return w.small_periodic(2, 8, 3, 1) if kind == "periodic" else w.small_sphere(2, 8, 3, 2)


def _field(h, f, seed=0):
    n = h.ni >> f
    G = n + 2
    return np.random.default_rng(123 + f + 1000 * seed).standard_normal((h.nblocks, G, G, G))


def _worker(rank, world, port, q):
    # one OpenMP thread per rank: the oracle's block loops are short here, and
    # idle threads of several ranks spinning between them only slow them down
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="1")
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
            ex = sharding.HaloExchange(h, owner, rank, n)
            a = _field(h, f)
            a[owner != rank] = np.nan          # another rank's blocks are unknown here
            t = torch.from_numpy(a.reshape(-1))   # shares memory with a
            for L in range(h.nlev):
                for d in range(3):
                    ex.ghost(t, L, d)
                    oracle_ghost_pass(h, a, f, L, d, cubic)
            mine = owner == rank
            q.put((rank, kind, f, cubic, a[mine].copy(), int(mine.sum()),
                   sum(ex.bytes_per_step().values())))
        for part in PARTS:
            for kind, f in OP_CASES:
                h = _hier(kind)
                owner = _owner(h, part, world)
                u, res, maxima = _split_operator(h, f, owner, rank)
                q.put((rank, "op", (kind, f, part), u[owner == rank].copy(), res[owner == rank].copy(), maxima))
            for kind in VMG_CASES:
                h = _hier(kind)
                owner = _owner(h, part, world)
                fine, base = _split_vmg(h, owner, rank)
                q.put((rank, "vmg", (kind, part), fine[owner == rank].copy(), base[owner == rank].copy()))
        for part in PARTS:
            h = _hier("periodic")
            q.put((rank, "mean", part, _split_mean(h, _owner(h, part, world), rank)))
        for kind, part in SOLVE_CASES:
            h = _solve_hier(kind)
            owner = _owner(h, part, world)
            rc, psi, g, st = _split_solve(h, owner, rank, kind)
            mine = owner == rank
            q.put((rank, "solve", (kind, part), rc, psi[mine].copy(), g[mine].copy(), st.outer_iters,
                   st.rho_mean, list(st.ratio)[:st.outer_iters], st.true_rel_residual))
        q.put((rank, "max", sharding.allreduce_max(float(rank + 1))))
    finally:
        dist.destroy_process_group()


def _split_operator(h, f, owner, rank):
    """SWEEPS red-black sweeps and then one residual of the composite
    operator on this rank's blocks, exchanges before the pieces that read
    other ranks' blocks; returns (u, residual, per-sweep maxima)."""
    import torch
    from code_only_b200 import sharding
    from tests import oracle_lib as ol
    n = h.ni >> f
    ex = sharding.HaloExchange(h, owner, rank, n)
    own = owner == rank
    u = _field(h, f)
    rhs = _field(h, f, seed=1)
    u[~own] = np.nan
    flux = [np.full_like(u, np.nan) for _ in range(3)]
    ut = torch.from_numpy(u.reshape(-1))
    ft = [torch.from_numpy(a.reshape(-1)) for a in flux]

    def poisson_flux():   # fmg_poisson_flux (fmg_poisson.F90:53-124)
        for Lc in range(h.nlev - 2, -1, -1):
            ex.converge(ut, Lc)
            ol.oracle_step(h, ol.STEP_CONVERGE, f, u=u, L=Lc, own=own)
        ol.oracle_step(h, ol.STEP_BOUNDARY_U, f, u=u, own=own)
        for L in range(h.nlev):
            for d in range(3):
                ex.ghost(ut, L, d)
                ol.oracle_step(h, ol.STEP_GHOST, f, u=u, L=L, d=d, own=own)
        ol.oracle_step(h, ol.STEP_BOUNDARY_U, f, u=u, own=own)
        ol.oracle_step(h, ol.STEP_FLUX, f, u=u, flux=flux, own=own)
        for d in range(3):
            ex.reflux(ft[d], d)
        ol.oracle_step(h, ol.STEP_FLUXCORR, f, flux=flux, own=own)

    maxima = []
    for _ in range(SWEEPS):
        m = 0.0
        for ipass in (1, 2):
            poisson_flux()
            out = np.zeros(1)
            ol.oracle_step(h, ol.STEP_RELAX, f, u=u, flux=flux, rhs=rhs, out=out, flag=ipass, own=own)
            m = max(m, float(out[0]))
        maxima.append(sharding.allreduce_max(m))
    poisson_flux()
    res = np.full_like(u, np.nan)
    ol.oracle_step(h, ol.STEP_RESID, f, flux=flux, rhs=rhs, out=res, own=own)
    return u, res, maxima


def _fmax(h):
    f = 0
    while (2 << f) < h.ni:
        f += 1
    return f


def _bc(kind):
    from code_only_b200 import abi
    return abi.SFM_BC_PERIODIC if kind == "periodic" else abi.SFM_BC_SPHERE


def _split_vmg(h, owner, rank):
    """The V-cycle's prolongation onto every AMR level and the base-grid
    solve on this rank's blocks, exchanges first; returns (prolonged field,
    field after the base solve)."""
    import torch
    from code_only_b200 import sharding
    from tests import oracle_lib as ol
    f = _fmax(h)
    ex = sharding.HaloExchange(h, owner, rank, h.ni >> f)
    own = owner == rank
    c, fine = _field(h, f, seed=2), _field(h, f, seed=3)
    u, r = _field(h, f, seed=4), _field(h, f, seed=5)
    for a in (c, fine, u, r):
        a[~own] = np.nan
    ct, ut, rt = (torch.from_numpy(a.reshape(-1)) for a in (c, u, r))
    for Lf in range(1, h.nlev):
        ex.p2c(ct, Lf - 1)
        ol.oracle_step(h, ol.STEP_P2C, f, u=c, out=fine, L=Lf, own=own)
    ex.base(ut)
    ex.base(rt)
    bc = _bc("periodic" if (h.touch == 0).all() else "sphere")
    ol.oracle_step(h, ol.STEP_BASE_SOLVE, f, u=u, rhs=r, own=own, bc=bc)
    return fine, u


def _rho(h):
    G = h.ni + 4   # two io ghost layers
    return np.random.default_rng(77).standard_normal((h.nblocks, G, G, G)) + 1.0


def _split_mean(h, owner, rank):
    """The mean of 4 pi G rho over the leaf cells as fmg_make_physvar forms
    it (fmg_data_if.F90:59-82): per-block sums of this rank's leaf blocks
    (k, j, i order), gathered, then folded in block order."""
    import torch
    from code_only_b200 import abi, sharding
    ex = sharding.HaloExchange(h, owner, rank, h.ni)
    four_pi_g = abi.default_params(abi.SFM_BC_PERIODIC).four_pi_G
    rho, n = _rho(h), h.ni
    part = np.full(h.nblocks, np.nan)
    leaf = h.child[:, 0] < 0
    for b in np.nonzero((owner == rank) & leaf)[0]:
        s = 0.0
        for k in range(n):
            for j in range(n):
                for i in range(n):
                    s = s + float(rho[b, k + 2, j + 2, i + 2]) * four_pi_g
        part[b] = s
    part = ex.gather_blocks(torch.from_numpy(part)).numpy()
    mass = vol = 0.0
    for b in np.nonzero(leaf)[0]:   # blocks are sorted by level
        hL = float(h.cellwidth[h.level[b]])
        dv = hL * hL * hL
        mass = mass + float(part[b]) * dv
        vol = vol + float(n * n * n) * dv
    return mass / vol


# whole-solve cases: (boundary, owners); the isolated boundaries gather the
# base blocks for their moments, the z-periodic cylinder for its line density
SOLVE_CASES = [("periodic", "morton"), ("periodic", "alternating"), ("periodic", "nested"),
               ("sphere", "alternating"), ("zmirror", "alternating"), ("cylinder", "alternating")]


def _solve_hier(kind):
    from code_only_b200 import workloads as w
    if kind == "zmirror":
        return w.mirror_sphere(2, 8, 3)
    if kind == "cylinder":
        return w.zperiodic_cylinder(2, 8, 3)
    return _hier(kind)


def _solve_params(kind="periodic"):
    from code_only_b200 import abi
    bc = {"periodic": abi.SFM_BC_PERIODIC, "sphere": abi.SFM_BC_SPHERE, "zmirror": abi.SFM_BC_ZMIRROR,
          "cylinder": abi.SFM_BC_CYL_ZPERIODIC}[kind]
    kw = {} if kind == "periodic" else {"zero_mean": 0}
    # two outer iterations on the periodic box, one or two elsewhere (each
    # rank's exchanges go through gloo: a split solve costs seconds per
    # iteration)
    return abi.default_params(bc, rel_tol=1e-3 if kind == "periodic" else 0.5, max_outer=40, **kw)


def _solve_rho(h, kind="periodic"):
    from code_only_b200 import abi, workloads as w
    fn = {"periodic": w.gaussian_peak, "sphere": w.softened_sphere, "zmirror": w.wide_sphere,
          "cylinder": w.beaded_line}[kind]
    return w.block_field(h, abi.default_params(abi.SFM_BC_PERIODIC).ngh_io, fn)


def _split_solve(h, owner, rank, kind="periodic"):
    """The oracle's whole solve (fmg_cycle: set-up, outer loop of fmg_lin with
    the AMR-level V-cycle and the base-grid solve, psi and g) on this rank's
    blocks, every cross-rank read through the exchanges above; the blocks
    another rank owns start as NaN in rho and psi."""
    import torch
    from code_only_b200 import sharding
    from tests import oracle_lib as ol
    fmax = _fmax(h)
    ex = [sharding.HaloExchange(h, owner, rank, h.ni >> f) for f in range(fmax + 1)]
    rho = _solve_rho(h, kind)
    rho[owner != rank] = np.nan

    def exchanges(kind, f, L, d, a):
        t = torch.from_numpy(a)
        if kind == 0:
            ex[f].ghost(t, L, d)
        elif kind == 1:
            ex[f].converge(t, L, bool(d))
        elif kind == 2:
            ex[f].reflux(t, d)
        elif kind == 3:
            ex[f].p2c(t, L)
        elif kind == 4:
            ex[f].base(t)
        elif kind == 5:
            a[0] = sharding.allreduce_max(float(a[0]))
        elif kind == 6:
            a[:] = ex[0].gather_blocks(t).numpy()
        else:
            raise ValueError(f"unknown exchange kind {kind}")

    return ol.oracle_solve_split(h, rho, _solve_params(kind), owner, rank, exchanges)


def _run(world=2, timeout=900):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = []
    t0 = time.time()
    n_msgs = len(CASES) + len(PARTS) * (len(OP_CASES) + len(VMG_CASES) + 1) + len(SOLVE_CASES) + 1
    while len(out) < world * n_msgs and time.time() - t0 < timeout:
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


def test_nested_partition_keeps_subtrees_together():
    """partition(nested=True): every block on its parent's rank, so neither
    the restriction nor the prolongation between levels crosses ranks; the
    base level is cut by subtree weight."""
    from code_only_b200 import sharding, workloads as w
    for h in (_hier("periodic"), _hier("sphere"), w.nested_sphere(5, 8, 8)):
        for world in (2, 3, 4):
            owner = sharding.partition(h, world, nested=True)
            up = h.level > 0
            assert np.array_equal(owner[up], owner[h.parent[up]])
            assert set(np.unique(owner)) == set(range(world))
            for rank in range(world):
                ex = sharding.HaloExchange(h, owner, rank, h.ni)
                assert not any(k[0] in ("converge", "p2c") and v for k, v in ex.bytes_per_step().items())


def test_hilbert_key_is_a_hilbert_curve():
    """hilbert_key orders the points of a 2^b cube as a Hilbert curve: every
    point once, each step to a face neighbour, starting at the origin."""
    from code_only_b200.sharding import hilbert_key
    for bits in (1, 2, 3, 4):
        n = 1 << bits
        g = np.array([(i, j, k) for k in range(n) for j in range(n) for i in range(n)])
        key = hilbert_key(g, bits)
        assert sorted(key.tolist()) == list(range(n ** 3))
        pts = g[np.argsort(key)]
        assert (pts[0] == 0).all()
        assert (np.abs(np.diff(pts, axis=0)).sum(axis=1) == 1).all()


def test_hilbert_partitions_are_balanced():
    from code_only_b200 import sharding, workloads as w
    for h in (_hier("periodic"), w.nested_sphere(5, 8, 8)):
        for world in (2, 3, 4):
            o = sharding.partition(h, world, curve="hilbert")
            for L in range(h.nlev):
                c = np.bincount(o[h.level == L], minlength=world)
                assert c.max() - c.min() <= 1
            on = sharding.partition(h, world, nested=True, curve="hilbert")
            up = h.level > 0
            assert np.array_equal(on[up], on[h.parent[up]])
            assert set(np.unique(on)) == set(range(world))


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
           [x for x in two_ranks if x[1] not in ("max", "op", "vmg", "mean", "solve")] if (k, ff, c) == case}
    assert set(got) == {0, 1}, "a rank did not report"
    for r in (0, 1):
        assert np.isfinite(got[r]).all()
        assert np.array_equal(got[r], ref[owner == r])


def test_allreduce_max(two_ranks):
    vals = [x[2] for x in two_ranks if x[1] == "max"]
    assert vals == [2.0, 2.0]


def _single_rank_operator(h, f):
    """The same sweeps by the oracle's integrated fmg_poisson_relax, then the
    residual of the result (one rank, every block)."""
    from tests import oracle_lib as ol
    u = _field(h, f)
    rhs = _field(h, f, seed=1)
    maxima = [ol.oracle_relax(h, u, rhs, f, 1) for _ in range(SWEEPS)]
    flux = [np.zeros_like(u) for _ in range(3)]
    v = u   # the residual's fill updates u's ghost layers and covered cells, as in the split run
    # residual pieces without an ownership mask: fill, fluxes, correction
    for Lc in range(h.nlev - 2, -1, -1):
        ol.oracle_step(h, ol.STEP_CONVERGE, f, u=v, L=Lc)
    ol.oracle_step(h, ol.STEP_BOUNDARY_U, f, u=v)
    ol.oracle_ghost_pass(h, v, f, -1, 0, False)
    ol.oracle_step(h, ol.STEP_BOUNDARY_U, f, u=v)
    ol.oracle_step(h, ol.STEP_FLUX, f, u=v, flux=flux)
    ol.oracle_step(h, ol.STEP_FLUXCORR, f, flux=flux)
    res = np.zeros_like(u)
    ol.oracle_step(h, ol.STEP_RESID, f, flux=flux, rhs=rhs, out=res)
    return u, res, maxima


@pytest.mark.parametrize("part", PARTS)
@pytest.mark.parametrize("case", OP_CASES, ids=[f"{k}-f{f}" for k, f in OP_CASES])
def test_two_rank_relax_and_residual_are_bitwise(two_ranks, case, part):
    """Sweeps and residual of the composite operator split over two ranks
    (converge, ghost-pass and flux-correction exchanges) equal one rank's."""
    kind, f = case
    h = _hier(kind)
    u_ref, res_ref, max_ref = _single_rank_operator(h, f)
    owner = _owner(h, part)
    got = {x[0]: x[3:] for x in two_ranks if x[1] == "op" and x[2] == (kind, f, part)}
    assert set(got) == {0, 1}, "a rank did not report"
    for r in (0, 1):
        u, res, maxima = got[r]
        mine = owner == r
        assert np.isfinite(u).all()
        assert np.array_equal(u, u_ref[mine])
        skip = (h.level != h.nlev - 1) & (h.child[:, 0] >= 0)
        assert np.array_equal(res[~skip[mine]], res_ref[mine & ~skip])
        assert maxima == max_ref


def test_residual_pieces_match_the_composite_operator():
    """The pieces of oracle_step, run on one rank, give the oracle's own
    composite operator L u (oracle_apply_L: residual of rhs = 0)."""
    import ctypes as C
    from code_only_b200 import abi
    from tests import oracle_lib as ol
    h = _hier("periodic")
    u = _field(h, 0)
    v = u.copy()
    flux = [np.zeros_like(u) for _ in range(3)]
    for Lc in range(h.nlev - 2, -1, -1):
        ol.oracle_step(h, ol.STEP_CONVERGE, 0, u=v, L=Lc)
    ol.oracle_step(h, ol.STEP_BOUNDARY_U, 0, u=v)
    ol.oracle_ghost_pass(h, v, 0, -1, 0, False)
    ol.oracle_step(h, ol.STEP_BOUNDARY_U, 0, u=v)
    ol.oracle_step(h, ol.STEP_FLUX, 0, u=v, flux=flux)
    ol.oracle_step(h, ol.STEP_FLUXCORR, 0, flux=flux)
    res = np.zeros_like(u)
    ol.oracle_step(h, ol.STEP_RESID, 0, flux=flux, rhs=np.zeros_like(u), out=res)
    lu = np.zeros_like(u)
    lib = ol.load_oracle()
    rc = lib.oracle_apply_L(abi.HierDesc(h).ref(), C.byref(abi.default_params(abi.SFM_BC_PERIODIC)),
                            u.ctypes.data, lu.ctypes.data)
    assert rc == 0
    skip = (h.level != h.nlev - 1) & (h.child[:, 0] >= 0)
    assert np.array_equal(-res[~skip], lu[~skip])


def _drop_worker(rank, world, port, drop, q):
    """_split_operator on the periodic hierarchy with one kind of exchange
    turned into a no-op; reports whether the owned blocks stayed finite."""
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      OMP_NUM_THREADS="1")
    import datetime

    import torch.distributed as dist
    from code_only_b200 import sharding
    setattr(sharding.HaloExchange, drop, lambda *a, **k: None)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        h = _hier("periodic")
        owner = _owner(h, "alternating", world)
        if drop in ("p2c", "base"):
            a, b = _split_vmg(h, owner, rank)
        else:
            a, b = _split_operator(h, 0, owner, rank)[:2]
        q.put((rank, bool(np.isfinite(a[owner == rank]).all() and np.isfinite(b[owner == rank]).all())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("drop", ["ghost", "converge", "reflux", "p2c", "base"])
def test_dropping_an_exchange_leaves_unknown_values(drop):
    """Each kind of exchange is needed: without it a rank reads another rank's
    block that it never received (NaN here)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_drop_worker, args=(r, 2, port, drop, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        out = sorted(q.get(timeout=180) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    assert len(out) == 2 and not any(finite for _, finite in out)


@pytest.mark.parametrize("part", PARTS)
@pytest.mark.parametrize("kind", VMG_CASES)
def test_two_rank_vcycle_transfers_are_bitwise(two_ranks, kind, part):
    """The AMR-level V-cycle's prolongation (parent block to the child's
    owner) and base-grid solve (every base block to every rank) split over
    two ranks equal one rank's, block for block."""
    from tests import oracle_lib as ol
    h = _hier(kind)
    f = _fmax(h)
    c, fine = _field(h, f, seed=2), _field(h, f, seed=3)
    u, r = _field(h, f, seed=4), _field(h, f, seed=5)
    for Lf in range(1, h.nlev):
        ol.oracle_step(h, ol.STEP_P2C, f, u=c, out=fine, L=Lf)
    ol.oracle_step(h, ol.STEP_BASE_SOLVE, f, u=u, rhs=r, bc=_bc(kind))
    owner = _owner(h, part)
    got = {x[0]: x[3:] for x in two_ranks if x[1] == "vmg" and x[2] == (kind, part)}
    assert set(got) == {0, 1}, "a rank did not report"
    for rk in (0, 1):
        g_fine, g_base = got[rk]
        mine = owner == rk
        assert np.array_equal(g_fine, fine[mine])
        assert np.array_equal(g_base, u[mine])
        base = h.level[mine] == 0
        assert np.isfinite(g_base[base]).all()


@pytest.mark.parametrize("part", PARTS)
def test_two_rank_mean_is_bitwise(two_ranks, part):
    """Per-block sums gathered exactly and folded in block order give the
    oracle's own mean of 4 pi G rho (the solve's rho_mean) to the bit."""
    from code_only_b200 import abi
    from tests import oracle_lib as ol
    h = _hier("periodic")
    rc, _, _, st, _ = ol.oracle_solve(h, _rho(h), abi.default_params(abi.SFM_BC_PERIODIC), want_g=False)
    assert rc in (abi.SFM_OK, abi.SFM_ENOTCONVERGED)
    got = [x[3] for x in two_ranks if x[1] == "mean" and x[2] == part]
    assert len(got) == 2
    assert got[0] == got[1] == st.rho_mean


@pytest.mark.parametrize("case", SOLVE_CASES, ids=[f"{k}-{p}" for k, p in SOLVE_CASES])
def test_two_rank_solve_is_bitwise(two_ranks, case):
    """The whole FMG solve split over two ranks -- the oracle's fmg_cycle on
    each rank's blocks, every read of the other rank's blocks through the
    exchanges, maxima all-reduced, ordered sums gathered -- gives the
    single-rank solve bit for bit: psi and g on every owned block, the
    iteration count, the mean, the residual history."""
    from tests import oracle_lib as ol
    kind, part = case
    h = _solve_hier(kind)
    rc0, psi0, g0, st0, _ = ol.oracle_solve(h, _solve_rho(h, kind), _solve_params(kind))
    owner = _owner(h, part)
    got = {x[0]: x[3:] for x in two_ranks if x[1] == "solve" and x[2] == case}
    assert set(got) == {0, 1}, "a rank did not report"
    for r in (0, 1):
        rc, psi, g, iters, mean, ratios, trr = got[r]
        mine = owner == r
        assert rc == rc0
        assert iters == st0.outer_iters and mean == st0.rho_mean
        assert ratios == list(st0.ratio)[:st0.outer_iters]
        assert trr == st0.true_rel_residual
        assert np.array_equal(psi, psi0[mine])
        assert np.array_equal(g, g0[mine])



def _three_rank_worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      OMP_NUM_THREADS="1")
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        h = _hier("sphere")
        owner = _owner(h, "alternating", world)
        u, res, maxima = _split_operator(h, 0, owner, rank)
        q.put((rank, u[owner == rank].copy(), res[owner == rank].copy(), maxima))
    finally:
        dist.destroy_process_group()


def test_three_rank_relax_and_residual_are_bitwise():
    """The same exchanges with three ranks (blocks dealt round-robin, so a
    block's neighbours, parent and children mostly sit on two other ranks)."""
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_three_rank_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        got = {r: (u, res, m) for r, u, res, m in (q.get(timeout=300) for _ in procs)}
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    h = _hier("sphere")
    u_ref, res_ref, max_ref = _single_rank_operator(h, 0)
    owner = _owner(h, "alternating", world)
    skip = (h.level != h.nlev - 1) & (h.child[:, 0] >= 0)
    for r in range(world):
        u, res, maxima = got[r]
        mine = owner == r
        assert np.array_equal(u, u_ref[mine])
        assert np.array_equal(res[~skip[mine]], res_ref[mine & ~skip])
        assert maxima == max_ref
