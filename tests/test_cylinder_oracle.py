"""The z-periodic cylinder boundaries in the oracle
(fmg_boundary_phys_cyl_zperiodic.F90 and fmg_boundary_phys_mask_zperiodic.F90):
the box wraps in z and is isolated in x and y, where the first ghost layer
holds the 2D potential a00 ln(r) of the masked source's line density.

Checks against physics and the reference's formulas rather than against
the oracle itself: a source independent of z gives a potential independent
of z; the returned potential's ghost layer on the x and y faces equals
a00 ln(sqrt(x^2+y^2)) with a00 = (sum of 4 pi G rho dv over the base
level, after the mask) / zlen / (2 pi); the density mask zeroes exactly the
cells whose source is below rho_mask."""
import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from tests.oracle_lib import oracle_solve


def _solve(fn, bc, rho_mask=0.0, nlev=3):
    h = w.zperiodic_cylinder(2, 8, nlev)
    p = abi.default_params(bc, rel_tol=1e-10, max_outer=40, zero_mean=0, rho_mask=rho_mask)
    rho = w.block_field(h, p.ngh_io, fn)
    rc, psi, g, st, _ = oracle_solve(h, rho, p)
    assert rc == abi.SFM_OK and st.converged and st.true_rel_residual <= 1e-10
    return h, p, rho, psi


def test_line_mass_potential_is_independent_of_z():
    h, _, _, psi = _solve(w.line_mass, abi.SFM_BC_CYL_ZPERIODIC)
    n = h.ni
    a = psi[:, 2:2 + n, 2:2 + n, 2:2 + n]
    assert np.abs(a - a[:, :1]).max() <= 1e-12 * np.abs(a).max()
    # the same (level, x, y) column at every z holds the same values
    cols = {}
    for b in range(h.nblocks):
        cols.setdefault((int(h.level[b]), *np.round(h.x0[b, :2], 9)), []).append(b)
    for bs in cols.values():
        assert np.abs(a[bs] - a[bs[:1]]).max() <= 1e-12 * np.abs(a).max()


@pytest.mark.parametrize("bc,mask", [(abi.SFM_BC_CYL_ZPERIODIC, 0.0),
                                     (abi.SFM_BC_MASK_ZPERIODIC, 4 * np.pi * 0.05)])
def test_ghost_layer_is_the_line_potential(bc, mask):
    h, p, rho, psi = _solve(w.beaded_line, bc, mask)
    n, cw = h.ni, h.cellwidth
    src = p.four_pi_G * rho[:, 1:n + 3, 1:n + 3, 1:n + 3]    # (-1:n)^3 of every block
    xs, ys, zs = w.cell_centres(h, 1)
    if bc == abi.SFM_BC_CYL_ZPERIODIC:
        ext = [h.x0[h.level == 0][:, d] for d in range(2)]
        xmin, ymin = ext[0].min(), ext[1].min()
        xmax, ymax = ext[0].max() + (n - 1) * cw[0], ext[1].max() + (n - 1) * cw[0]
        rad2 = min(xmax, ymax, -xmin, -ymin) ** 2
        masked = (xs[:, None, None, :] ** 2 + ys[:, None, :, None] ** 2 + 0 * zs[:, :, None, None]) >= rad2
    else:
        masked = src < mask
    # the solve restricts the source onto covered cells before the boundary
    # (fmg_converge_c2p, fmg.F90:167): finest level first, the 8-mean
    src = src.copy()
    hn = n // 2
    for L in range(h.nlev - 1, 0, -1):
        for c in np.where(h.level == L)[0]:
            par = h.parent[c]
            o = h.ijk[c] % 2
            fine = src[c, 1:n + 1, 1:n + 1, 1:n + 1]
            mean = fine.reshape(hn, 2, hn, 2, hn, 2).mean(axis=(1, 3, 5))
            src[par, 1 + o[2] * hn:1 + (o[2] + 1) * hn, 1 + o[1] * hn:1 + (o[1] + 1) * hn,
                1 + o[0] * hn:1 + (o[0] + 1) * hn] = mean
    src = np.where(masked, 0.0, src)
    base = np.where(h.level == 0)[0]
    a00 = 0.0
    for b in base:   # the reference's order: base blocks, then k, j, i
        for v in src[b, 1:n + 1, 1:n + 1, 1:n + 1].ravel():
            a00 = a00 + v * cw[0] ** 3
    zmin = h.x0[base, 2].min()
    zmax = h.x0[base, 2].max() + (n - 1) * cw[0]
    a00 = a00 / (zmax - zmin + cw[0]) / (2.0 * (4.0 * np.arctan(1.0)))
    # x-min faces: ghost plane i = -1 (io index 1) over j, k in (-1:n)
    for b in np.where(h.touch[:, 0] == 1)[0]:
        x = xs[b, 0]
        y = ys[b, :]
        want = np.log(np.sqrt(x * x + y * y)) * a00
        got = psi[b, 1:n + 3, 1:n + 3, 1]
        assert np.allclose(got, np.broadcast_to(want, got.shape), rtol=1e-12, atol=0)
