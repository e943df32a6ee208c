"""Block links built on the device (sfm_link_blocks) against the host's.

workloads.build_hierarchy links every hierarchy on the host (the role of the
reference's grid.F90:587-731 link updates); sfm_link_blocks must give the
same parent, child, nbr and touch arrays from the blocks' levels and
positions alone -- for periodic, isolated and partly periodic boxes, for
blocks in any order, and it must report malformed block sets."""
import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from code_only_b200.solver import SFMError, link_blocks

pytestmark = pytest.mark.gpu

HIERARCHIES = {
    "amr3_periodic": lambda: w.small_periodic(2, 8, 3, 1),
    "amr3_sphere": lambda: w.small_sphere(2, 8, 3, 2),
    "uniform64": lambda: w.uniform_periodic(8, 8),
    "nested5": lambda: w.nested_sphere(5, 8, 8),
    "zmirror_base3": lambda: w.mirror_sphere(3, 8, 3),
    "cylinder_zperiodic": lambda: w.zperiodic_cylinder(2, 8, 3),
}


def _periodic(h):
    """per-direction periodicity as the hierarchy's links show it: a
    direction is periodic when no face along it touches the boundary"""
    return [not h.touch[:, 2 * d:2 * d + 2].any() for d in range(3)]


def _device_links(h, order=None):
    import torch
    lev = np.asarray(h.level, dtype=np.int32)
    ijk = np.asarray(h.ijk, dtype=np.int32)
    if order is not None:
        lev, ijk = lev[order], ijk[order]
    out = link_blocks(torch.from_numpy(lev).cuda(), torch.from_numpy(ijk).cuda(), h.ngb, _periodic(h), h.nlev)
    return [t.cpu().numpy() for t in out]


@pytest.mark.parametrize("name", list(HIERARCHIES))
def test_device_links_equal_the_host_links(name):
    h = HIERARCHIES[name]()
    parent, child, nbr, touch = _device_links(h)
    assert np.array_equal(parent, h.parent)
    assert np.array_equal(child, h.child)
    assert np.array_equal(nbr, h.nbr)
    assert np.array_equal(touch, h.touch)


def test_any_block_order():
    """Blocks given in a shuffled order: every link names the same block,
    renumbered by the shuffle."""
    h = HIERARCHIES["amr3_sphere"]()
    order = np.random.default_rng(5).permutation(h.nblocks)
    inv = np.empty_like(order)
    inv[order] = np.arange(h.nblocks)
    parent, child, nbr, touch = _device_links(h, order)
    ren = lambda a: np.where(a >= 0, inv[np.maximum(a, 0)], -1)
    assert np.array_equal(parent, ren(h.parent[order]))
    assert np.array_equal(child, ren(h.child[order]))
    assert np.array_equal(nbr, ren(h.nbr[order]))
    assert np.array_equal(touch, h.touch[order])


def test_links_feed_sfm_create():
    """A context created from device-built links solves exactly as one from
    the host's (FP64 bit-identical)."""
    import dataclasses
    from code_only_b200.solver import FMGPoisson
    h = HIERARCHIES["amr3_periodic"]()
    parent, child, nbr, touch = _device_links(h)
    h2 = dataclasses.replace(h, parent=parent.astype(np.int32), child=child.astype(np.int32),
                             nbr=nbr.astype(np.int32), touch=touch.astype(np.int8))
    p = abi.default_params(abi.SFM_BC_PERIODIC)
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    with FMGPoisson(h, params=p) as s:
        psi1, g1, _ = s.solve(rho)
    with FMGPoisson(h2, params=p) as s:
        psi2, g2, _ = s.solve(rho)
    assert np.array_equal(psi1, psi2) and np.array_equal(g1, g2)


def _expect_ehier(lev, ijk, ngb, periodic, nlev):
    import torch
    with pytest.raises(SFMError) as e:
        link_blocks(torch.tensor(lev, dtype=torch.int32).cuda(), torch.tensor(ijk, dtype=torch.int32).cuda(),
                    ngb, periodic, nlev)
    assert e.value.code == abi.SFM_EHIER


def test_malformed_block_sets_are_reported():
    base = [(i, j, k) for k in range(2) for j in range(2) for i in range(2)]
    kids = [(i, j, k) for k in range(2) for j in range(2) for i in range(2)]   # the 8 children of base block 0
    # a duplicated block
    _expect_ehier([0] * 9, base + [base[3]], (2, 2, 2), True, 1)
    # a block outside its level's box
    _expect_ehier([0] * 8, base[:7] + [(2, 0, 0)], (2, 2, 2), True, 1)
    # a child without its parent level's block (base block 0 missing)
    _expect_ehier([0] * 7 + [1] * 8, base[1:] + kids, (2, 2, 2), True, 2)
    # a parent with 7 of its 8 children
    _expect_ehier([0] * 8 + [1] * 7, base + kids[:7], (2, 2, 2), True, 2)
