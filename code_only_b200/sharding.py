"""Block partition and ghost-cell halo exchange across ranks (one GPU each).

The reference decomposes the hierarchy over MPI ranks block by block: each
rank owns the blocks of every AMR level that a Peano-Hilbert curve assigns
to it (refine.F90:662-706), and every ghost fill exchanges packed face
slabs with the ranks owning the neighbours (fmg_ghostcell.F90:162,168 for
same-level faces, :353,358 for coarse-fine ones).  This module is the same
step for GPU ranks:

* ``partition(h, world)`` -- the blocks of each AMR level are already in
  Morton order (workloads.build_hierarchy); each level is cut into `world`
  contiguous ranges of nearly equal block counts, so each rank owns a
  compact region on every level.
* ``HaloExchange`` -- for every step of the composite operator that reads
  across blocks, the cells a rank's own blocks read from blocks another
  rank owns:
  - each pass (AMR level L, direction d) of the three-pass ghost fill: the
    neighbour's boundary plane (whole transverse range, ghosts included) for
    a same-level face, the coarse block's layer (the octant's half face plus
    one cell on each side) for a coarse-fine face (fmg_ghostcell.F90:162,168,
    353,358);
  - each level of fmg_converge_c2p (children at L + 1 restricted onto their
    parent at L): the child's interior for the linear restriction, the whole
    block with its ghost layer for the cubic one (fmg_converge.F90:139,144);
  - the flux correction: the face fluxes of a fine block whose face borders
    the parent level, read by the owner of the coarse neighbour
    (fmg_reflux.F90:158,166);
  - the prolongation of the AMR-level V-cycle (vmg_interp_p2c_lev,
    vmg_interpol.F90:82-164): the whole parent block, read by the child's
    owner (the V-cycle's restriction is the converge step);
  - the base-grid solve (mg_dataPrepare, mg_data.F90:179-253): the interior
    of every base block, read by every rank, each of which then solves the
    base grid itself and keeps its own base blocks (the same gather serves
    the isolated boundary's multipole moments, one running sum over the
    base cells in order, evaluated by every rank);
  - ordered sums (``gather_blocks``): per-block partials gathered exactly,
    then folded in block order on every rank.
  Both ends derive the same lists from the hierarchy, so a step's exchange
  is one grouped send/receive per peer of the packed values
  (``torch.distributed`` P2P: gloo between CPU ranks, NCCL between GPUs),
  each into the receiver's own copy of the sender's block -- never a load
  from another GPU's memory.

Run before each such step, the exchanges make a rank's owned blocks hold
exactly the values a single rank computes: after the ghost fill, after
whole red-black sweeps and residuals of the composite operator, after the
V-cycle's prolongation and base-grid solve, and through a whole FMG solve
(tests/test_sharding.py, world size 2, bit for bit, for Morton-range and
alternating owners).  Residual maxima are an
all-reduce of one value (``allreduce_max``); the base grid (at most 32^3
cells) is gathered whole on every rank, where the base-grid solve runs
redundantly.
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

__all__ = ["partition", "hilbert_key", "HaloExchange", "allreduce_max"]


def hilbert_key(ijk: np.ndarray, bits: int) -> np.ndarray:
    """Index of each integer point (int [m, 3], 0 <= coordinate < 2^bits)
    along the 3-D Hilbert curve, the curve the reference deals blocks to
    ranks along (its Peano-Hilbert fillcells, refine.F90:662-706).  The
    transform is Skilling's (Programming the Hilbert curve, AIP Conf. Proc.
    707, 2004): axes to transposed index, then the bits interleaved."""
    X = [np.asarray(ijk[:, d], dtype=np.int64).copy() for d in range(3)]
    M = 1 << (bits - 1)
    Q = M
    while Q > 1:   # inverse undo of the rotations and reflections
        P = Q - 1
        for i in range(3):
            hi = (X[i] & Q) != 0
            X[0] = np.where(hi, X[0] ^ P, X[0])
            t = np.where(hi, 0, (X[0] ^ X[i]) & P)
            X[0] ^= t
            X[i] ^= t
        Q >>= 1
    for i in range(1, 3):   # Gray encode
        X[i] ^= X[i - 1]
    t = np.zeros_like(X[0])
    Q = M
    while Q > 1:
        t = np.where((X[2] & Q) != 0, t ^ (Q - 1), t)
        Q >>= 1
    for i in range(3):
        X[i] ^= t
    key = np.zeros_like(X[0])
    for bit in range(bits - 1, -1, -1):
        for i in range(3):
            key = (key << 1) | ((X[i] >> bit) & 1)
    return key


def _curve_order(h, s: int, e: int, curve: str) -> np.ndarray:
    """block ids s..e-1 (one AMR level, stored in Morton order) in the order
    of the chosen space-filling curve"""
    ids = np.arange(s, e, dtype=np.int64)
    if curve == "morton":
        return ids
    if curve != "hilbert":
        raise ValueError(f"unknown curve {curve!r}")
    ijk = np.asarray(h.ijk[s:e], dtype=np.int64)
    bits = max(1, int(ijk.max()).bit_length()) if e > s else 1
    return ids[np.argsort(hilbert_key(ijk, bits), kind="stable")]


def partition(h, world: int, nested: bool = False, curve: str = "morton") -> np.ndarray:
    """owner[nb]: rank of every block.

    Default: the blocks of each AMR level cut into `world` consecutive runs
    of nearly equal block counts along a space-filling curve (Morton, or
    Hilbert as the reference deals its blocks, refine.F90:662-706).  nested:
    the base level is cut along the curve into runs of nearly equal weight
    (a base block weighs as many blocks as its subtree holds) and every
    block inherits its parent's rank, so the restriction and the
    prolongation between levels stay on one rank and only faces between
    subtrees cross ranks -- at the price of whole subtrees as the unit of
    balance."""
    if world < 1:
        raise ValueError("world must be >= 1")
    owner = np.empty(h.nblocks, dtype=np.int32)
    starts = np.concatenate([[0], np.cumsum(h.level_counts())]).astype(np.int64)
    if nested:
        weight = np.ones(h.nblocks, dtype=np.int64)
        for b in range(h.nblocks - 1, int(starts[1]) - 1, -1):   # children come after their parents
            weight[h.parent[b]] += weight[b]
        order = _curve_order(h, 0, int(starts[1]), curve)
        cum = np.concatenate([[0], np.cumsum(weight[order])])
        target = cum[-1] * np.arange(1, world, dtype=np.int64) / world
        cuts = np.concatenate([[0], np.searchsorted(cum[1:], target, side="left") + 1, [order.size]])
        for r in range(world):
            owner[order[cuts[r]:cuts[r + 1]]] = r
        for b in range(int(starts[1]), h.nblocks):
            owner[b] = owner[h.parent[b]]
        return owner
    for L in range(h.nlev):
        s, e = int(starts[L]), int(starts[L + 1])
        order = _curve_order(h, s, e, curve)
        cut = (np.arange(world + 1, dtype=np.int64) * (e - s)) // world
        for r in range(world):
            owner[order[cut[r]:cut[r + 1]]] = r
    return owner


def _faces(h):
    """(kind[nb,6], src[nb,6]): 0 same-level neighbour, 1 parent-level
    neighbour (coarse-fine face), 2 physical boundary; the source block."""
    nb = h.nblocks
    kind = np.full((nb, 6), 2, dtype=np.int8)
    src = np.full((nb, 6), -1, dtype=np.int64)
    same = h.nbr >= 0
    kind[same] = 0
    src[same] = h.nbr[same]
    for b in np.nonzero(h.level > 0)[0]:
        p = h.parent[b]
        for f in range(6):
            if kind[b, f] == 0 or h.touch[b, f]:
                continue
            q = h.nbr[p, f]
            if q >= 0:
                kind[b, f] = 1
                src[b, f] = q
    return kind, src


def _put3(d, x, a, b):
    return (x, a, b) if d == 0 else ((a, x, b) if d == 1 else (a, b, x))


class HaloExchange:
    """Send and receive lists of every cross-block step for one rank.

    Cell indices are flat offsets into a field (or face-flux array) of shape
    [nb, G, G, G] (G = n + 2, i fastest), the layout of one fmg level; every
    rank holds full-size arrays and owns the blocks ``owner == rank``.
    Steps are keyed ("ghost", L, d), ("converge", L, cubic), ("reflux", d),
    ("p2c", L) and ("base",).
    """

    def __init__(self, h, owner: np.ndarray, rank: int, n: int):
        self.h, self.owner, self.rank, self.n = h, np.asarray(owner), rank, n
        self._idx_cache = {}
        self.world = int(self.owner.max()) + 1
        G = n + 2
        self.G, self.V = G, G ** 3
        kind, src = _faces(h)
        lev = np.asarray(h.level)
        nb2 = n // 2
        # needs[step][(reader, holder)] -> sorted unique flat cells the
        # reader's blocks read from blocks the holder owns
        self.needs: Dict[tuple, Dict[Tuple[int, int], np.ndarray]] = {}
        rng = np.arange(-1, n + 1)
        for L in range(h.nlev):
            blocks = np.nonzero(lev == L)[0]
            for d in range(3):
                acc: Dict[Tuple[int, int], List[np.ndarray]] = {}
                for b in blocks:
                    reader = int(self.owner[b])
                    for lr in range(2):
                        f = lr + 2 * d
                        k = kind[b, f]
                        if k == 2:
                            continue
                        s = int(src[b, f])
                        holder = int(self.owner[s])
                        if holder == reader:
                            continue
                        if k == 0:   # the neighbour's boundary plane, whole transverse range
                            xs = n - 1 if lr == 0 else 0
                            pa, qa = np.meshgrid(rng, rng, indexing="xy")
                        else:        # the coarse layer: octant half face +- 1 cell
                            if L == 0:
                                continue
                            xs = n - 1 if lr == 0 else 0
                            ta = 1 if d == 0 else 0
                            tb = 1 if d == 2 else 2
                            oa, ob = int(h.ijk[b, ta] & 1) * nb2, int(h.ijk[b, tb] & 1) * nb2
                            cr = np.arange(-1, nb2 + 1)
                            pa, qa = np.meshgrid(cr + oa, cr + ob, indexing="xy")
                        i, j, kk = _put3(d, xs, pa.ravel(), qa.ravel())
                        cells = s * self.V + ((kk + 1) * G + (j + 1)) * G + (i + 1)
                        acc.setdefault((reader, holder), []).append(np.asarray(cells, dtype=np.int64))
                self.needs[("ghost", L, d)] = {key: np.unique(np.concatenate(v)) for key, v in acc.items()}
        # converge_c2p of level Lc: the parent's owner reads its children
        inner = np.arange(0, n)
        whole = np.arange(-1, n + 1)
        for Lc in range(h.nlev - 1):
            for cubic in (False, True):
                r = whole if cubic else inner
                kk, jj, ii = np.meshgrid(r, r, r, indexing="ij")
                off = (((kk + 1) * G + (jj + 1)) * G + (ii + 1)).ravel()
                acc = {}
                for b in np.nonzero(lev == Lc + 1)[0]:
                    reader, holder = int(self.owner[h.parent[b]]), int(self.owner[b])
                    if reader != holder:
                        acc.setdefault((reader, holder), []).append(int(b) * self.V + off)
                self.needs[("converge", Lc, cubic)] = {k: np.unique(np.concatenate(v)) for k, v in acc.items()}
        # flux correction: a fine face next to the parent level is read by the
        # coarse neighbour's owner (the n x n fluxes on that face)
        pq = np.arange(0, n)
        pa, qa = np.meshgrid(pq, pq, indexing="xy")
        for d in range(3):
            acc = {}
            for b in np.nonzero(lev > 0)[0]:
                for lr in range(2):
                    f = lr + 2 * d
                    if kind[b, f] != 1:
                        continue
                    reader, holder = int(self.owner[src[b, f]]), int(self.owner[b])
                    if reader == holder:
                        continue
                    xf = -1 if lr == 0 else n - 1
                    i, j, kk = _put3(d, xf, pa.ravel(), qa.ravel())
                    acc.setdefault((reader, holder), []).append(
                        int(b) * self.V + ((kk + 1) * G + (j + 1)) * G + (i + 1))
            self.needs[("reflux", d)] = {k: np.unique(np.concatenate(v)) for k, v in acc.items()}
        # prolongation of the AMR-level V-cycle (vmg_interp, parent onto its
        # children at Lc + 1): the child's owner reads the whole parent block,
        # ghost layer included (the trilinear stencil reaches it)
        kk, jj, ii = np.meshgrid(whole, whole, whole, indexing="ij")
        whole_off = (((kk + 1) * G + (jj + 1)) * G + (ii + 1)).ravel()
        for Lc in range(h.nlev - 1):
            acc = {}
            for b in np.nonzero(lev == Lc + 1)[0]:
                p = int(h.parent[b])
                reader, holder = int(self.owner[b]), int(self.owner[p])
                if reader != holder:
                    acc.setdefault((reader, holder), []).append(p * self.V + whole_off)
            self.needs[("p2c", Lc)] = {k: np.unique(np.concatenate(v)) for k, v in acc.items()}
        # base-grid solve (vmg_slvsml -> mg_dataPrepare): every rank gathers
        # the interiors of all base blocks and solves the base grid itself
        kk, jj, ii = np.meshgrid(inner, inner, inner, indexing="ij")
        inner_off = (((kk + 1) * G + (jj + 1)) * G + (ii + 1)).ravel()
        acc = {}
        for b in np.nonzero(lev == 0)[0]:
            holder = int(self.owner[b])
            for reader in range(self.world):
                if reader != holder:
                    acc.setdefault((reader, holder), []).append(int(b) * self.V + inner_off)
        self.needs[("base",)] = {k: np.unique(np.concatenate(v)) for k, v in acc.items()}

    def ghost(self, field, L: int, d: int):
        """Exchange before ghost pass (L, d) of `field`."""
        self.exchange(field, ("ghost", L, d))

    def converge(self, field, Lc: int, cubic: bool = False):
        """Exchange before converge_c2p of level Lc (children at Lc + 1)."""
        self.exchange(field, ("converge", Lc, bool(cubic)))

    def reflux(self, flux_d, d: int):
        """Exchange of direction d's face fluxes before the flux correction."""
        self.exchange(flux_d, ("reflux", d))

    def p2c(self, field, Lc: int):
        """Exchange before the prolongation of level Lc onto Lc + 1."""
        self.exchange(field, ("p2c", Lc))

    def base(self, field):
        """Exchange before the base-grid solve: every base block to every rank."""
        self.exchange(field, ("base",))

    def gather_blocks(self, values):
        """Every block's value of a per-block array ([nb] float64 torch
        tensor, this rank's entries set) from its owner: an all-reduce sum
        in which every other rank adds -0.0, so each entry comes out exactly
        as its owner had it (signed zeros and NaN included).  The ordered
        sums of the solve -- the mean of rho (fmg_data_if.F90:59-82) and the
        level averages of vmg_zeroAverage -- then fold these per-block
        partials in block order on every rank, the single-rank order."""
        import torch
        import torch.distributed as dist
        mine = torch.from_numpy(self.owner == self.rank).to(values.device)
        t = torch.where(mine, values, torch.full_like(values, -0.0))
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return t

    def exchange(self, field, step: tuple):
        """Send the values of this rank's blocks that other ranks read in
        `step`, receive the values this rank reads from theirs, each into
        this rank's copy of the sender's block.  `field` is a flat contiguous
        torch tensor (CPU with gloo, CUDA with NCCL); every rank calls this
        for every step in the same order."""
        import torch
        import torch.distributed as dist
        ops, recvs = [], []
        for (reader, holder), cells in self.needs.get(step, {}).items():
            if self.rank not in (reader, holder):
                continue
            idx = self._index(step, reader, holder, cells, field.device)
            if holder == self.rank:
                ops.append(dist.P2POp(dist.isend, field[idx].contiguous(), reader))
            elif reader == self.rank:
                buf = torch.empty(cells.size, dtype=field.dtype, device=field.device)
                ops.append(dist.P2POp(dist.irecv, buf, holder))
                recvs.append((idx, buf))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for idx, buf in recvs:
            field[idx] = buf

    def _index(self, step, reader, holder, cells, device):
        """the cell list as an index tensor on `device`, made once per step
        and device (on a GPU, one upload instead of one per exchange)"""
        import torch
        key = (step, reader, holder, str(device))
        idx = self._idx_cache.get(key)
        if idx is None:
            idx = torch.from_numpy(cells).to(device)
            self._idx_cache[key] = idx
        return idx

    def bytes_per_step(self) -> Dict[tuple, int]:
        """Values this rank receives per step x 8 bytes (FP64)."""
        out = {}
        for key, m in self.needs.items():
            out[key] = 8 * sum(int(c.size) for (reader, _), c in m.items() if reader == self.rank)
        return out


def allreduce_max(value: float, device=None) -> float:
    """Max over ranks of one value (the residual maxima of fmg_poisson.F90:212)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
