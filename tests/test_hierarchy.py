"""Hierarchy generation and the link-list invariants of fmg_check_linklist
(fmg_data_if.F90:415-568), including host-side fault injection: a corrupted
hierarchy must be refused with SFM_EHIER by both the oracle and the CUDA
library's sfm_create (which validates on the host before touching a GPU)."""
import ctypes as C

import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from tests.oracle_lib import load_oracle


def check(h):
    return load_oracle().oracle_check_linklist(abi.HierDesc(h).ref())


def product_create(sfmg_lib, h, **kw):
    p = abi.default_params(**kw)
    ctx = C.c_void_p()
    rc = sfmg_lib.sfm_create(abi.HierDesc(h).ref(), C.byref(p), C.byref(ctx))
    if rc == 0:
        sfmg_lib.sfm_destroy(ctx)
    return rc


GENERATORS = {
    "uniform": lambda: w.uniform_periodic(4, 8),
    "nested5": lambda: w.nested_sphere(5, 8, 8),
    "nested3_periodic": lambda: w.nested_sphere(3, 4, 8, periodic=True),
    "random_periodic": lambda: w.small_periodic(4, 8, 4, 11),
    "random_sphere": lambda: w.small_sphere(4, 8, 4, 12),
}


@pytest.mark.parametrize("name", list(GENERATORS))
def test_generated_hierarchies_satisfy_invariants(name):
    h = GENERATORS[name]()
    assert check(h) == abi.SFM_OK
    # proper nesting: every refined block has all 26 neighbours on its level
    for L in range(1, h.nlev):
        lv = h.ijk[h.level == L]
        keys = {tuple(v) for v in lv.tolist()}
        ext = np.array(h.ngb) << L
        for q in h.ijk[(h.level == L) & (h.child[:, 0] >= 0)]:
            for d in np.ndindex(3, 3, 3):
                nbq = q + np.array(d) - 1
                if h.periodic:
                    nbq = np.mod(nbq, ext)
                elif np.any(nbq < 0) or np.any(nbq >= ext):
                    continue
                assert tuple(nbq) in keys


def test_config2_structure():
    h = w.nested_sphere()
    assert h.nblocks == 2560 and list(h.level_counts()) == [512] * 5
    assert int(h.leaf_mask().sum()) == 2304 and h.leaf_cells() == 2304 * 512
    assert np.all(h.touch[h.level == 0].sum(axis=1) <= 3)
    assert h.touch[h.level > 0].sum() == 0


def test_periodic_links_wrap():
    h = w.uniform_periodic(4, 8)
    assert h.touch.sum() == 0 and np.all(h.nbr >= 0)
    # the left x-neighbour of i=0 is i=3 on the same j,k
    b = int(np.where((h.ijk == [0, 1, 2]).all(axis=1))[0][0])
    n = h.nbr[b, 0]
    assert list(h.ijk[n]) == [3, 1, 2]


def _corruptions(h0):
    """(label, hierarchy) pairs, each breaking one invariant."""
    out = []
    h = w.small_periodic(2, 8, 3, 5)
    fine = np.where(h.level == 2)[0]
    b = int(fine[0])
    # 1. neighbour symmetry broken
    c = w.Hierarchy(**{**h.__dict__})
    c.nbr = h.nbr.copy()
    f = int(np.where(c.nbr[b] >= 0)[0][0])
    c.nbr[b, f] = int(fine[1]) if c.nbr[b, f] != fine[1] else int(fine[2])
    out.append(("asymmetric neighbour", c))
    # 2. child -> parent -> self broken
    c = w.Hierarchy(**{**h.__dict__})
    c.parent = h.parent.copy()
    c.parent[b] = int(c.parent[int(fine[-1])]) if c.parent[int(fine[-1])] != c.parent[b] else 0
    out.append(("wrong parent", c))
    # 3. a face with both a neighbour and the physical boundary
    c = w.Hierarchy(**{**h.__dict__})
    c.touch = h.touch.copy()
    c.touch[b, f] = 1
    out.append(("neighbour and boundary", c))
    # 4. level order broken
    c = w.Hierarchy(**{**h.__dict__})
    c.level = h.level.copy()
    c.level[0], c.level[-1] = c.level[-1], c.level[0]
    out.append(("unsorted levels", c))
    # 5. a face of a fine block left without any link (missing parent-level neighbour)
    hs = w.small_sphere(2, 8, 2, 0)
    c = w.Hierarchy(**{**hs.__dict__})
    c.nbr = hs.nbr.copy()
    c.touch = hs.touch.copy()
    base = np.where(hs.level == 0)[0]
    bb = int(base[0])
    fb = int(np.where(hs.nbr[bb] >= 0)[0][0])
    other = int(hs.nbr[bb, fb])
    c.nbr[bb, fb] = -1
    c.nbr[other, fb ^ 1] = -1
    out.append(("dangling face", c))
    return out


@pytest.mark.parametrize("idx", range(5))
def test_corrupted_hierarchy_is_refused_by_oracle(idx):
    label, c = _corruptions(None)[idx]
    assert check(c.contiguous()) == abi.SFM_EHIER, label


@pytest.mark.parametrize("idx", range(5))
def test_corrupted_hierarchy_is_refused_by_library(sfmg_lib, idx):
    label, c = _corruptions(None)[idx]
    assert product_create(sfmg_lib, c.contiguous()) == abi.SFM_EHIER, label


def test_grf_statistics():
    rho = w.gaussian_random_field(32, 12345, kmax=16.0)
    assert abs(rho.mean() - 1.0) < 1e-12
    assert abs(np.log(rho).std() - 1.5) < 1e-9
