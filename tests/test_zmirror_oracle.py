"""The z-mirror boundary (fmg_boundary_phys_zmirror.F90) in the oracle,
checked against physics rather than against itself: for a density even in
z, the solve on the box's upper half with the mirror plane on its z-min face
must give the potential of the ordinary isolated solve on the mirror-
symmetric double box.  The two discrete problems are the same: the mirror
ghost u(:,:,-1) = u(:,:,0) is what the symmetric solution holds across
z = 0, the half box's moments carry the mirror's factors 2 and 0 (equal to
the full box's moments, which have no odd-in-z part), and both boxes mask
the density at the same radius.  Base boxes of 3^3 and 3 x 3 x 6 blocks
(not powers of two) take the reference's base-level sweeps in both."""
import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from tests.oracle_lib import oracle_solve


def _pair(nlev):
    hh = w.mirror_sphere(3, 8, nlev)
    hf = w.mirror_sphere(3, 8, nlev, full=True)
    up = np.where(hf.x0[:, 2] > 0)[0]
    key = {(int(hh.level[b]), *np.round(hh.x0[b], 9)): b for b in range(hh.nblocks)}
    idx = np.array([key[(int(hf.level[b]), *np.round(hf.x0[b], 9))] for b in up])
    return hh, hf, up, idx


@pytest.mark.parametrize("nlev", [2, 3])
def test_mirror_half_box_equals_symmetric_full_box(nlev):
    hh, hf, up, idx = _pair(nlev)
    assert len(up) * 2 == hf.nblocks and len(idx) == hh.nblocks   # the full box mirrors the half
    out = {}
    for name, h, bc in (("half", hh, abi.SFM_BC_ZMIRROR), ("full", hf, abi.SFM_BC_SPHERE)):
        p = abi.default_params(bc, rel_tol=1e-11, max_outer=40, zero_mean=0, lmax=3)
        rho = w.block_field(h, p.ngh_io, w.wide_sphere)
        rc, psi, g, st, _ = oracle_solve(h, rho, p)
        assert rc == abi.SFM_OK and st.converged
        out[name] = (psi, g)
    n = hh.ni
    a = out["half"][0][idx][:, 2:2 + n, 2:2 + n, 2:2 + n]
    b = out["full"][0][up][:, 2:2 + n, 2:2 + n, 2:2 + n]
    assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    ga = out["half"][1][idx][:, :, 2:2 + n, 2:2 + n, 2:2 + n]
    gb = out["full"][1][up][:, :, 2:2 + n, 2:2 + n, 2:2 + n]
    assert np.abs(ga - gb).max() / np.abs(gb).max() <= 1e-9


def test_mirror_ghost_layer_mirrors_the_first_plane():
    """After the solve, psi's ghost plane below every block on the mirror
    face equals its first interior plane (fmg_restore_u returns U with its
    ghost layer)."""
    hh = w.mirror_sphere(3, 8, 2)
    p = abi.default_params(abi.SFM_BC_ZMIRROR, rel_tol=1e-10, max_outer=30, zero_mean=0)
    rho = w.block_field(hh, p.ngh_io, w.wide_sphere)
    rc, psi, _, _, _ = oracle_solve(hh, rho, p)
    assert rc == abi.SFM_OK
    on = np.where(hh.touch[:, 4] == 1)[0]
    assert on.size > 0
    # (k, j, i) axes with 2 io ghost layers: plane k = -1 is index 1, k = 0 index 2
    assert np.array_equal(psi[on, 1, 1:-1, 1:-1], psi[on, 2, 1:-1, 1:-1])


def test_mhd_be_sphere_masks_at_the_cloud_radius():
    """fmg_boundary_phys_sphere_MHD_BE.F90 is the sphere module with the mask
    radius Rcloud: with r_cloud equal to the sphere module's own radius
    min(xmax, ymax, zmax, -xmin, -ymin, -zmin) the solve is the sphere's to
    the bit; a smaller cloud masks more of the source."""
    h = w.small_sphere(2, 8, 3, 2)
    n = h.ni
    base = h.x0[h.level == 0]
    cw = h.cellwidth[0]
    rr = min(base[:, 0].max() + (n - 1) * cw, base[:, 1].max() + (n - 1) * cw, base[:, 2].max() + (n - 1) * cw,
             -base[:, 0].min(), -base[:, 1].min(), -base[:, 2].min())
    kw = dict(rel_tol=1e-10, max_outer=30, zero_mean=0)
    rho = w.block_field(h, 2, w.softened_sphere)
    _, psi_s, _, _, _ = oracle_solve(h, rho, abi.default_params(abi.SFM_BC_SPHERE, **kw))
    _, psi_b, _, _, _ = oracle_solve(h, rho, abi.default_params(abi.SFM_BC_SPHERE_MHD_BE, r_cloud=rr, **kw))
    assert np.array_equal(psi_s, psi_b)
    rc, psi_c, _, st, _ = oracle_solve(h, rho, abi.default_params(abi.SFM_BC_SPHERE_MHD_BE, r_cloud=0.2, **kw))
    assert rc == abi.SFM_OK and st.converged
    assert not np.array_equal(psi_c, psi_s)
