"""Synthetic block-structured AMR hierarchies and densities.

The reference builds its hierarchy with its own refinement machinery
(refine.F90, refineCond_nest_jeans.F90) and hands the Poisson solver a fixed
octree of NI^3 blocks.  This module produces the same kind of octree from a
refinement predicate, in the numbering the solver's C ABI expects
(blocks sorted by AMR level; faces lr + 2*dir; children lri + 2*lrj + 4*lrk),
together with seeded densities at cell centres:

* ``uniform_periodic``   -- one level, periodic (64^3 box as 8^3 blocks)
* ``nested_sphere``      -- concentric levels, each covering the central half
                            of its parent, isolated boundary
* ``jeans_cloud``        -- log-normal Gaussian random field refined by the
                            Jeans rule of refineCond_nest_jeans.F90:66-105
* ``small_*``            -- tiny hierarchies for parity tests

Proper nesting is enforced across all 26 neighbours: a block is refined only
when every neighbour of it exists on its level, which guarantees that a
parent-level link always ends one level up (the assumption behind
fmg_ghfix_parentlev, fmg_ghostcell.F90:350).
"""
from __future__ import annotations

import dataclasses
import math
import os
from concurrent.futures import ThreadPoolExecutor
from typing import Callable, Optional, Sequence

import numpy as np

__all__ = [
    "Hierarchy", "build_hierarchy", "uniform_periodic", "nested_sphere",
    "jeans_cloud", "small_periodic", "small_sphere", "cell_centres",
    "block_field", "config_hierarchy",
]


@dataclasses.dataclass
class Hierarchy:
    ni: int                     # cells per block edge
    ngb: tuple                  # base blocks per dimension
    nlev: int                   # AMR levels present
    periodic: bool
    box_lo: np.ndarray          # (3,)
    box_size: float
    level: np.ndarray           # int32 [nb]
    ijk: np.ndarray             # int32 [nb,3]
    parent: np.ndarray          # int32 [nb]
    child: np.ndarray           # int32 [nb,8]
    nbr: np.ndarray             # int32 [nb,6]
    touch: np.ndarray           # int8  [nb,6]
    cellwidth: np.ndarray       # float64 [nlev]
    x0: np.ndarray              # float64 [nb,3] centre of cell (0,0,0)

    @property
    def nblocks(self) -> int:
        return int(self.level.shape[0])

    def level_counts(self):
        return np.bincount(self.level, minlength=self.nlev)

    def leaf_mask(self):
        return self.child[:, 0] < 0

    def leaf_cells(self) -> int:
        return int(self.leaf_mask().sum()) * self.ni ** 3

    def contiguous(self) -> "Hierarchy":
        for f in ("level", "ijk", "parent", "child", "nbr"):
            setattr(self, f, np.ascontiguousarray(getattr(self, f), dtype=np.int32))
        self.touch = np.ascontiguousarray(self.touch, dtype=np.int8)
        self.cellwidth = np.ascontiguousarray(self.cellwidth, dtype=np.float64)
        self.x0 = np.ascontiguousarray(self.x0, dtype=np.float64)
        return self


def _morton(ijk: np.ndarray) -> np.ndarray:
    """Interleaved-bit key of (i,j,k) (i lowest), for block ordering."""
    key = np.zeros(ijk.shape[0], dtype=np.int64)
    for bit in range(20):
        for d in range(3):
            key |= ((ijk[:, d].astype(np.int64) >> bit) & 1) << (3 * bit + d)
    return key


def _pack(ijk: np.ndarray) -> np.ndarray:
    ijk = ijk.astype(np.int64)
    return (ijk[:, 2] << 42) | (ijk[:, 1] << 21) | ijk[:, 0]


_NEIGH26 = np.array([(a, b, c) for c in (-1, 0, 1) for b in (-1, 0, 1) for a in (-1, 0, 1)
                     if (a, b, c) != (0, 0, 0)], dtype=np.int64)


def build_hierarchy(ngb: Sequence[int], ni: int, nlev: int,
                    refine: Callable[[int, np.ndarray, "Hierarchy"], np.ndarray],
                    periodic, box_lo=(0.0, 0.0, 0.0), box_size: float = 1.0,
                    max_iter: int = 50) -> Hierarchy:
    """Builds a properly nested octree.

    ``periodic``: one bool for all three directions, or three (x, y, z);
    a periodic direction wraps its links, the others touch the physical
    boundary.

    ``refine(level, ijk, geom)`` returns a bool mask over the blocks ``ijk``
    (int array [m,3]) of ``level``: True refines the block into 8 children.
    ``geom`` carries ``ni``, ``box_lo``, ``box_size`` and ``ngb`` for the
    predicate to compute cell coordinates.
    """
    ngb = tuple(int(v) for v in ngb)
    per = (bool(periodic),) * 3 if np.isscalar(periodic) else tuple(bool(v) for v in periodic)
    periodic = all(per)
    box_lo = np.asarray(box_lo, dtype=np.float64)
    geom = Hierarchy(ni=ni, ngb=ngb, nlev=nlev, periodic=periodic, box_lo=box_lo,
                     box_size=float(box_size), level=None, ijk=None, parent=None,
                     child=None, nbr=None, touch=None, cellwidth=None, x0=None)
    forced = [set() for _ in range(nlev)]
    for _ in range(max_iter):
        levels = []
        flags = []
        cur = np.array([(i, j, k) for k in range(ngb[2]) for j in range(ngb[1]) for i in range(ngb[0])],
                       dtype=np.int64)
        for L in range(nlev):
            levels.append(cur)
            if L == nlev - 1:
                flags.append(np.zeros(cur.shape[0], dtype=bool))
                break
            f = np.asarray(refine(L, cur, geom), dtype=bool).copy()
            if forced[L]:
                key = _pack(cur)
                fk = np.fromiter(forced[L], dtype=np.int64)
                f |= np.isin(key, fk)
            flags.append(f)
            par = cur[f]
            if par.shape[0] == 0:
                break
            off = np.array([(a, b, c) for c in (0, 1) for b in (0, 1) for a in (0, 1)], dtype=np.int64)
            cur = (2 * par[:, None, :] + off[None, :, :]).reshape(-1, 3)
        # proper nesting: every neighbour of a refined block must exist
        changed = False
        for L in range(1, len(levels)):
            if L >= len(flags) or not flags[L].any():
                continue
            ext = np.array(ngb, dtype=np.int64) << L
            blk = levels[L]
            keyset = np.sort(_pack(blk))
            ref = blk[flags[L]]
            nb_ = (ref[:, None, :] + _NEIGH26[None, :, :]).reshape(-1, 3)
            for d in range(3):
                if per[d]:
                    nb_[:, d] = np.mod(nb_[:, d], ext[d])
            ok = np.all((nb_ >= 0) & (nb_ < ext), axis=1)
            nb_ = nb_[ok]
            k = _pack(nb_)
            pos = np.searchsorted(keyset, k)
            pos = np.minimum(pos, keyset.size - 1)
            missing = nb_[keyset[pos] != k]
            if missing.shape[0]:
                par = np.unique(_pack(missing // 2))
                new = set(par.tolist()) - forced[L - 1]
                if new:
                    forced[L - 1] |= new
                    changed = True
        if not changed:
            break
    else:
        raise RuntimeError("nesting did not converge")
    levels = [lv for lv in levels if lv.shape[0] > 0]
    nlev_eff = len(levels)
    # order blocks: level-major, Morton within level
    order_lv = []
    for L, lv in enumerate(levels):
        o = np.argsort(_morton(lv), kind="stable")
        order_lv.append(lv[o])
    counts = [lv.shape[0] for lv in order_lv]
    starts = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    nb = int(starts[-1])
    level = np.concatenate([np.full(c, L, dtype=np.int32) for L, c in enumerate(counts)])
    ijk = np.concatenate(order_lv).astype(np.int64)
    keys = [_pack(lv) for lv in order_lv]
    sorted_keys = [np.argsort(k) for k in keys]

    def lookup(L, q):
        """global ids of blocks q (int64 [m,3]) on level L, -1 if absent"""
        out = np.full(q.shape[0], -1, dtype=np.int64)
        if L < 0 or L >= nlev_eff or q.shape[0] == 0:
            return out
        ks = keys[L][sorted_keys[L]]
        kq = _pack(q)
        pos = np.searchsorted(ks, kq)
        pos = np.minimum(pos, ks.size - 1)
        hit = ks[pos] == kq
        out[hit] = sorted_keys[L][pos[hit]] + starts[L]
        return out

    parent = np.full(nb, -1, dtype=np.int64)
    child = np.full((nb, 8), -1, dtype=np.int64)
    nbr = np.full((nb, 6), -1, dtype=np.int64)
    touch = np.zeros((nb, 6), dtype=np.int8)
    for L in range(nlev_eff):
        s, e = starts[L], starts[L + 1]
        q = ijk[s:e]
        if L > 0:
            parent[s:e] = lookup(L - 1, q // 2)
        if L + 1 < nlev_eff:
            for c in range(8):
                off = np.array([c & 1, (c >> 1) & 1, (c >> 2) & 1], dtype=np.int64)
                child[s:e, c] = lookup(L + 1, 2 * q + off)
        ext = np.array(ngb, dtype=np.int64) << L
        for d in range(3):
            for lr in (0, 1):
                off = np.zeros(3, dtype=np.int64)
                off[d] = -1 if lr == 0 else 1
                qq = q + off
                edge = (qq[:, d] < 0) | (qq[:, d] >= ext[d])
                if per[d]:
                    qq = np.mod(qq, ext)
                    nbr[s:e, lr + 2 * d] = lookup(L, qq)
                else:
                    res = np.full(q.shape[0], -1, dtype=np.int64)
                    inside = ~edge
                    res[inside] = lookup(L, qq[inside])
                    nbr[s:e, lr + 2 * d] = res
                    touch[s:e, lr + 2 * d] = edge.astype(np.int8)
    # a block either has all 8 children or none
    has = child >= 0
    if not np.all(has.all(axis=1) | (~has).all(axis=1)):
        raise RuntimeError("partial refinement")
    cw = np.array([box_size / (ngb[0] * ni * (1 << L)) for L in range(nlev_eff)], dtype=np.float64)
    x0 = box_lo[None, :] + (ijk.astype(np.float64) * ni + 0.5) * cw[level][:, None]
    h = Hierarchy(ni=ni, ngb=ngb, nlev=nlev_eff, periodic=periodic, box_lo=box_lo,
                  box_size=float(box_size), level=level, ijk=ijk.astype(np.int32),
                  parent=parent.astype(np.int32), child=child.astype(np.int32),
                  nbr=nbr.astype(np.int32), touch=touch, cellwidth=cw, x0=x0)
    return h.contiguous()


def cell_centres(h: Hierarchy, ngh: int):
    """Coordinates [nb, (ni+2g)] per axis of every cell incl. ghosts."""
    idx = np.arange(-ngh, h.ni + ngh, dtype=np.float64)
    cw = h.cellwidth[h.level]
    xs = h.x0[:, 0:1] + idx[None, :] * cw[:, None]
    ys = h.x0[:, 1:2] + idx[None, :] * cw[:, None]
    zs = h.x0[:, 2:3] + idx[None, :] * cw[:, None]
    return xs, ys, zs


def _threads() -> int:
    return max(1, min(32, os.cpu_count() or 1))


def block_field(h: Hierarchy, ngh: int, fn: Callable) -> np.ndarray:
    """Evaluates fn(x,y,z) at every cell centre (ghosts included), returning
    [nb, G, G, G] with axes (k, j, i) -- i fastest in memory.  Chunks of
    blocks are evaluated on a thread pool (elementwise: same values)."""
    xs, ys, zs = cell_centres(h, ngh)
    G = h.ni + 2 * ngh
    out = np.empty((h.nblocks, G, G, G), dtype=np.float64)
    chunk = 2048

    def part(s):
        e = min(s + chunk, h.nblocks)
        v = fn(xs[s:e, None, None, :], ys[s:e, None, :, None], zs[s:e, :, None, None])
        out[s:e] = np.broadcast_to(v, (e - s, G, G, G))

    with ThreadPoolExecutor(_threads()) as ex:
        list(ex.map(part, range(0, h.nblocks, chunk)))
    return out


# ---------------------------------------------------------------------------
# configurations
# ---------------------------------------------------------------------------
def uniform_periodic(nbase: int = 8, ni: int = 8) -> Hierarchy:
    """One level, periodic: (nbase*ni)^3 cells in a unit box."""
    return build_hierarchy((nbase,) * 3, ni, 1, lambda L, q, g: np.zeros(q.shape[0], bool), True,
                           box_lo=(0.0, 0.0, 0.0), box_size=1.0)


def _central_half(L, q, g: Hierarchy):
    """refine the blocks of level L lying in the central half of level L's
    extent: level L >= 1 spans ngb blocks per axis around the domain centre,
    so its central half is ngb/2 blocks wide"""
    ext = np.array(g.ngb, dtype=np.int64) << L
    half = np.maximum(np.array(g.ngb) // 4, 1)
    c = ext // 2
    return np.all((q >= c - half) & (q < c + half), axis=1)


def nested_sphere(nlev: int = 5, nbase: int = 8, ni: int = 8, periodic: bool = False) -> Hierarchy:
    """Base (nbase*ni)^3 in [-1/2,1/2]^3 plus nlev-1 concentric levels, each
    covering the central half of its parent (nbase^3 blocks per level)."""
    return build_hierarchy((nbase,) * 3, ni, nlev, _central_half, periodic,
                           box_lo=(-0.5, -0.5, -0.5), box_size=1.0)


def small_periodic(nbase: int = 2, ni: int = 8, nlev: int = 2, seed: int = 0) -> Hierarchy:
    """A few blocks with a seeded refinement pattern, periodic."""
    rng = np.random.default_rng(seed)

    def ref(L, q, g):
        m = rng.random(q.shape[0]) < 0.35
        if not m.any():
            m[rng.integers(0, q.shape[0])] = True
        return m

    return build_hierarchy((nbase,) * 3, ni, nlev, ref, True, box_lo=(0.0, 0.0, 0.0), box_size=1.0)


def small_sphere(nbase: int = 2, ni: int = 8, nlev: int = 2, seed: int = 0) -> Hierarchy:
    rng = np.random.default_rng(seed)

    def ref(L, q, g):
        m = rng.random(q.shape[0]) < 0.35
        if not m.any():
            m[rng.integers(0, q.shape[0])] = True
        return m

    return build_hierarchy((nbase,) * 3, ni, nlev, ref, False, box_lo=(-0.5, -0.5, -0.5), box_size=1.0)


def _near_origin(levels_radius):
    """Refines a block when the point of its box nearest the origin lies
    within levels_radius[L] (a predicate symmetric under z -> -z)."""
    def ref(L, q, g):
        cw = g.box_size / (g.ngb[0] * g.ni * (1 << L))
        lo = g.box_lo[None, :] + q * g.ni * cw
        hi = lo + g.ni * cw
        near = np.clip(0.0, lo, hi)
        return np.sqrt((near * near).sum(axis=1)) < levels_radius[min(L, len(levels_radius) - 1)]
    return ref


def mirror_sphere(nbase: int = 3, ni: int = 8, nlev: int = 3, full: bool = False) -> Hierarchy:
    """An isolated box for the z-mirror boundary: [-1/2, 1/2]^2 x [0, 1] with
    nbase^3 base blocks (the mirror plane z = 0 is the box's z-min face),
    refined around the origin.  full=True gives the box's mirror-symmetric
    double [-1/2, 1/2]^2 x [-1, 1] (nbase x nbase x 2 nbase base blocks) for
    the ordinary isolated boundary: its upper half holds the same blocks."""
    radii = (0.3, 0.15, 0.08, 0.04)
    if full:
        return build_hierarchy((nbase, nbase, 2 * nbase), ni, nlev, _near_origin(radii), False,
                               box_lo=(-0.5, -0.5, -1.0), box_size=1.0)
    return build_hierarchy((nbase,) * 3, ni, nlev, _near_origin(radii), False,
                           box_lo=(-0.5, -0.5, 0.0), box_size=1.0)


def _near_axis(levels_radius):
    """Refines a block when the point of its box nearest the z axis lies
    within levels_radius[L] (independent of z)."""
    def ref(L, q, g):
        cw = g.box_size / (g.ngb[0] * g.ni * (1 << L))
        lo = g.box_lo[None, :2] + q[:, :2] * g.ni * cw
        hi = lo + g.ni * cw
        near = np.clip(0.0, lo, hi)
        return np.sqrt((near * near).sum(axis=1)) < levels_radius[min(L, len(levels_radius) - 1)]
    return ref


def zperiodic_cylinder(nbase: int = 2, ni: int = 8, nlev: int = 3) -> Hierarchy:
    """[-1/2, 1/2]^3 periodic in z, isolated in x and y (the box of
    fmg_boundary_phys_cyl_zperiodic.F90 and ..._mask_zperiodic.F90), with
    nbase^3 base blocks refined around the z axis."""
    return build_hierarchy((nbase,) * 3, ni, nlev, _near_axis((0.3, 0.15, 0.08, 0.04)), (False, False, True),
                           box_lo=(-0.5, -0.5, -0.5), box_size=1.0)


def line_mass(x, y, z):
    """rho = 1/(1+(R/0.08)^2) for R < 0.45, else 1e-3, R = sqrt(x^2+y^2):
    independent of z."""
    R = np.sqrt(x * x + y * y) + 0.0 * z
    return np.where(R < 0.45, 1.0 / (1.0 + (R / 0.08) ** 2), 1e-3)


def beaded_line(x, y, z):
    """line_mass modulated along z (period 1/2): a z-periodic source that
    depends on z."""
    return line_mass(x, y, z) * (1.0 + 0.5 * np.cos(4.0 * np.pi * z))


def wide_sphere(x, y, z):
    """rho = 1/(1+(r/0.08)^2) for r < 0.45, else 1e-3 (centred at the origin;
    even in z)."""
    r = np.sqrt(x * x + y * y + z * z)
    return np.where(r < 0.45, 1.0 / (1.0 + (r / 0.08) ** 2), 1e-3)


def gaussian_random_field(n: int, seed: int, kmin: float = 2.0, kmax: float = 64.0,
                          slope: float = -4.0, sigma: float = 1.5) -> np.ndarray:
    """ln(rho) on an n^3 periodic grid: P(k) ~ k^slope for kmin <= |k| <= kmax
    (k in units of the box's fundamental mode), normalised to std sigma; rho
    is normalised to mean 1.  Axes (z, y, x)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    kz = k1[:, None, None]
    ky = k1[None, :, None]
    kx = np.fft.rfftfreq(n, d=1.0 / n)[None, None, :]
    kk = np.sqrt(kx * kx + ky * ky + kz * kz)
    amp = np.zeros_like(kk)
    band = (kk >= kmin) & (kk <= kmax)
    amp[band] = kk[band] ** (slope / 2.0)
    noise = rng.standard_normal(kk.shape) + 1j * rng.standard_normal(kk.shape)
    field = np.fft.irfftn(noise * amp, s=(n, n, n), axes=(0, 1, 2))
    field = (field - field.mean()) / field.std() * sigma
    rho = np.exp(field)
    return rho / rho.mean()


def _trilinear_periodic(grid: np.ndarray, x, y, z):
    """Trilinear interpolation of a cell-centred periodic unit-box grid (axes z,y,x)."""
    n = grid.shape[0]
    fx, fy, fz = x * n - 0.5, y * n - 0.5, z * n - 0.5
    ix, iy, iz = np.floor(fx).astype(np.int64), np.floor(fy).astype(np.int64), np.floor(fz).astype(np.int64)
    tx, ty, tz = fx - ix, fy - iy, fz - iz
    out = 0.0
    for dz in (0, 1):
        wz = tz if dz else 1.0 - tz
        for dy in (0, 1):
            wy = ty if dy else 1.0 - ty
            for dx in (0, 1):
                wx = tx if dx else 1.0 - tx
                out = out + wz * wy * wx * grid[(iz + dz) % n, (iy + dy) % n, (ix + dx) % n]
    return out


def jeans_cloud(nlev: int = 6, nbase: int = 16, ni: int = 8, seed: int = 12345,
                cs: float = 0.2, jeans_const: float = 8.0, box_size: float = 6.0,
                cores: Optional[int] = None, core_seed: int = 99, core_rho: float = 1e6,
                core_a: float = 1e-4):
    """Jeans-refined turbulent cloud: ln(rho) a Gaussian random field on the
    (nbase*ni)^3 base grid, refined wherever a block has fewer than
    `jeans_const` cells per Jeans length cs*sqrt(pi/(G rho)) (G = 1,
    refineCond_nest_jeans.F90:90-103).  Finer levels sample rho by trilinear
    interpolation of the base field (plus optional Plummer cores).
    Returns (hierarchy, density function of (x,y,z))."""
    n = nbase * ni
    grid = gaussian_random_field(n, seed)
    centres = None
    if cores:
        rng = np.random.Generator(np.random.PCG64(core_seed))
        centres = rng.random((cores, 3))

    def rho_fn(x, y, z):
        u = np.mod(x / box_size, 1.0)
        v = np.mod(y / box_size, 1.0)
        w = np.mod(z / box_size, 1.0)
        r = _trilinear_periodic(grid, u, v, w)
        if centres is not None:
            for c in centres:
                dx = (np.mod(u - c[0] + 0.5, 1.0) - 0.5)
                dy = (np.mod(v - c[1] + 0.5, 1.0) - 0.5)
                dz = (np.mod(w - c[2] + 0.5, 1.0) - 0.5)
                r2 = dx * dx + dy * dy + dz * dz
                r = r + core_rho * (1.0 + r2 / (core_a * core_a)) ** -2.5
        return r

    def refine(L, q, g: Hierarchy):
        h = box_size / (nbase * ni * (1 << L))
        # block-max density on the block's cells, sampled at cell centres
        idx = (np.arange(ni) + 0.5) * h
        lo = q.astype(np.float64) * ni * h
        out = np.zeros(q.shape[0], dtype=bool)
        chunk = 512

        def part(s):
            qs = lo[s:s + chunk]
            xs = qs[:, 0:1] + idx[None, :]
            ys = qs[:, 1:2] + idx[None, :]
            zs = qs[:, 2:3] + idx[None, :]
            r = rho_fn(xs[:, None, None, :], ys[:, None, :, None], zs[:, :, None, None])
            rmax = r.reshape(r.shape[0], -1).max(axis=1)
            jlen = cs * np.sqrt(math.pi / rmax)
            out[s:s + chunk] = jlen < jeans_const * h

        with ThreadPoolExecutor(_threads()) as ex:   # elementwise per block: same decisions
            list(ex.map(part, range(0, q.shape[0], chunk)))
        return out

    h = build_hierarchy((nbase,) * 3, ni, nlev, refine, True, box_lo=(0.0, 0.0, 0.0), box_size=box_size)
    return h, rho_fn


def softened_sphere(x, y, z):
    """rho = 1/(1+(r/0.02)^2) for r < 0.4, else 1e-2 (box centred at 0)."""
    r = np.sqrt(x * x + y * y + z * z)
    return np.where(r < 0.4, 1.0 / (1.0 + (r / 0.02) ** 2), 1e-2)


def gaussian_peak(x, y, z):
    """rho = 1 + 100 exp(-r^2/(2*0.1^2)), r from the centre of the unit box."""
    r2 = (x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2
    return 1.0 + 100.0 * np.exp(-r2 / (2.0 * 0.1 ** 2))


def config_hierarchy(name: str):
    """(hierarchy, density fn, bc) for a named workload:
    'uniform64'  : 64^3 periodic, 8^3 blocks of 8^3, Gaussian peak
    'nested5'    : 64^3 base + 4 concentric levels, softened sphere, isolated
    'jeans6'     : 128^3 base periodic Jeans-refined GRF, 6 levels; the
                   box is 6 length units (G = 1, c_s = 0.2), the smallest size at
                   which this density reaches the sixth level: 133,856 blocks
    'deep8'      : 256^3 base of 16^3 blocks, 8 levels, GRF + Plummer cores
    'uniform256' : 256^3 periodic, 32^3 blocks of 8^3, Gaussian peak: the smallest
                   uniform grid whose FP32 field with ghosts (131 MB) exceeds the
                   126 MB L2, used for kernel profiles of the 8^3-block sweeps
    'uniform128' : 128^3 periodic, 16^3 blocks of 8^3: the smallest uniform grid
                   with jeans6's 32^3 base grid, used to profile the base-grid CTA
    'jeans3'     : the jeans6 density refined to 3 levels (89,800 blocks; the finest
                   level's FP32 field, 224 MB, exceeds L2): kernel profiles of
                   AMR-level operations at a few GB of device memory
    """
    if name == "uniform64":
        return uniform_periodic(8, 8), gaussian_peak, 0
    if name == "nested5":
        return nested_sphere(5, 8, 8), softened_sphere, 1
    if name == "uniform256":
        return uniform_periodic(32, 8), gaussian_peak, 0
    if name == "uniform128":
        return uniform_periodic(16, 8), gaussian_peak, 0
    if name == "jeans3":
        h, fn = jeans_cloud(nlev=3, nbase=16, ni=8)
        return h, fn, 0
    if name == "jeans6":
        h, fn = jeans_cloud(nlev=6, nbase=16, ni=8)
        return h, fn, 0
    if name == "deep8":
        h, fn = jeans_cloud(nlev=8, nbase=16, ni=16, cores=8, box_size=6.0)
        return h, fn, 0
    raise KeyError(name)
