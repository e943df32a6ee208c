"""The CPU restatement of the reference (oracle/) checked against known
answers.  The reference ships no golden vectors and cannot run here, so
these pin the restated operator and solver analytically:

* a periodic Fourier mode is an eigenvector of the 7-point operator with
  eigenvalue sum_d (2 cos(k h) - 2)/h^2: the solve must return it exactly;
* the composite coarse-fine operator (bilinear/bicubic transverse +
  quadratic normal ghosts, reflux) is exact on linear potentials: L(a.x) = 0;
* with a source manufactured as f = L(phi*), the FMG solve returns phi*;
* the multipole boundary converges to the direct sum with the order l;
* the stopping rule of fmg_cycle (fmg.F90:179-196).
"""
import ctypes as C

import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from tests.oracle_lib import load_oracle, oracle_solve


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_periodic_eigenmode_is_reproduced():
    h = w.uniform_periodic(2, 8)
    n = 16
    hh = 1.0 / n
    k = 2 * np.pi
    lam = (2 * np.cos(k * hh) - 2) / hh ** 2 + (2 * np.cos(2 * k * hh) - 2) / hh ** 2
    fn = lambda x, y, z: 1.0 + lam * np.sin(k * x) * np.cos(2 * k * y) / (4 * np.pi) + 0 * z
    p = abi.default_params(abi.SFM_BC_PERIODIC, rel_tol=1e-12, max_outer=30)
    rho = w.block_field(h, 2, fn)
    rc, psi, g, st, _ = oracle_solve(h, rho, p)
    assert rc == abi.SFM_OK
    exact = w.block_field(h, 2, lambda x, y, z: np.sin(k * x) * np.cos(2 * k * y) + 0 * z)
    a = psi[:, 2:10, 2:10, 2:10]
    e = exact[:, 2:10, 2:10, 2:10]
    assert rel(a - a.mean(), e - e.mean()) < 1e-11
    assert st.true_rel_residual < 1e-12
    # g = -grad phi from the face fluxes: the discrete derivative of the mode
    gx = g[:, 0, 2:10, 2:10, 2:10]
    xs, ys, zs = w.cell_centres(h, 2)
    X = xs[:, None, None, 2:10]
    Y = ys[:, None, 2:10, None]
    gx_exact = -(np.sin(k * (X + hh)) - np.sin(k * (X - hh))) / (2 * hh) * np.cos(2 * k * Y) + 0 * gx
    assert rel(gx, gx_exact) < 1e-10


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_composite_operator_exact_on_linear_potentials(seed):
    lib = load_oracle()
    h = w.small_sphere(2, 8, 3, seed)
    p = abi.default_params(abi.SFM_BC_SPHERE, zero_mean=0, ngh_io=1)
    phi = w.block_field(h, 1, lambda x, y, z: 0.3 * x - 1.7 * y + 0.9 * z + 0.25)
    out = np.zeros_like(phi)
    assert lib.oracle_apply_L(abi.HierDesc(h).ref(), C.byref(p), phi.ctypes.data, out.ctypes.data) == 0
    leaf = h.leaf_mask() | (h.level == h.nlev - 1)
    inner = out[leaf][:, 1:9, 1:9, 1:9]
    # operator values scale like 1/h^2: compare against |phi| / h_finest^2
    scale = np.abs(phi).max() / h.cellwidth[-1] ** 2
    assert np.abs(inner).max() / scale < 1e-13


@pytest.mark.parametrize("seed", [3, 4])
def test_manufactured_solution_is_recovered(seed):
    lib = load_oracle()
    h = w.small_periodic(2, 8, 3, seed)
    k = 2 * np.pi
    phi_fn = lambda x, y, z: np.sin(k * x) * np.cos(k * y) + 0.5 * np.sin(2 * k * z + 0.3)
    p1 = abi.default_params(abi.SFM_BC_PERIODIC, ngh_io=1)
    phi = w.block_field(h, 1, phi_fn)
    f = np.zeros_like(phi)
    assert lib.oracle_apply_L(abi.HierDesc(h).ref(), C.byref(p1), phi.ctypes.data, f.ctypes.data) == 0
    # leaves hold L(phi*); the solve restricts covered blocks from them
    rho = f / (4 * np.pi)
    p = abi.default_params(abi.SFM_BC_PERIODIC, ngh_io=1, rel_tol=1e-13, max_outer=40, stagnation_exit=0)
    rc, psi, g, st, _ = oracle_solve(h, rho, p)
    assert abs(st.rho_mean) < 1e-9            # the composite flux form conserves: sum L(phi) dV = 0
    leaf = h.leaf_mask() | (h.level == h.nlev - 1)
    a = psi[leaf][:, 1:9, 1:9, 1:9]
    e = phi[leaf][:, 1:9, 1:9, 1:9]
    assert rel(a - a.mean(), e - e.mean()) < 1e-9


def test_multipole_boundary_converges_with_order():
    lib = load_oracle()
    h = w.small_sphere(4, 8, 1, 0)            # 32^3 single level in [-1/2,1/2]^3
    p3 = abi.default_params(abi.SFM_BC_SPHERE, zero_mean=0, ngh_io=1, lmax=3)
    p4 = abi.default_params(abi.SFM_BC_SPHERE, zero_mean=0, ngh_io=1, lmax=4)
    c = [(0.11, -0.07, 0.05), (-0.09, 0.12, -0.1)]
    src_fn = lambda x, y, z: sum(np.exp(-((x - a) ** 2 + (y - b) ** 2 + (z - d) ** 2) / (2 * 0.04 ** 2))
                                 for a, b, d in c)
    src = w.block_field(h, 1, src_fn)
    rng = np.random.default_rng(7)
    pts = rng.normal(size=(64, 3))
    pts = pts / np.linalg.norm(pts, axis=1)[:, None] * 1.0
    out3 = np.zeros(64)
    out4 = np.zeros(64)
    d = abi.HierDesc(h)
    lib.oracle_multipole(d.ref(), C.byref(p3), src.ctypes.data, 64, pts.ctypes.data, out3.ctypes.data)
    lib.oracle_multipole(d.ref(), C.byref(p4), src.ctypes.data, 64, pts.ctypes.data, out4.ctypes.data)
    # direct sum over the base-level interior cells: phi = -1/(4 pi) sum src dV / |r - r'|
    xs, ys, zs = w.cell_centres(h, 1)
    X = np.broadcast_to(xs[:, None, None, 1:9], (h.nblocks, 8, 8, 8)).ravel()
    Y = np.broadcast_to(ys[:, None, 1:9, None], (h.nblocks, 8, 8, 8)).ravel()
    Z = np.broadcast_to(zs[:, 1:9, None, None], (h.nblocks, 8, 8, 8)).ravel()
    S = src[:, 1:9, 1:9, 1:9].ravel() * h.cellwidth[0] ** 3
    direct = np.array([-np.sum(S / np.sqrt((q[0] - X) ** 2 + (q[1] - Y) ** 2 + (q[2] - Z) ** 2)) / (4 * np.pi)
                       for q in pts])
    e3 = rel(out3, direct)
    e4 = rel(out4, direct)
    # truncation error ~ (r'/r)^(l+1): l = 4 must gain about one order over l = 3
    assert e3 < 1e-3 and e4 < e3 / 4


def test_stopping_rule_and_stagnation():
    h = w.small_periodic(2, 8, 2, 0)
    rho = w.block_field(h, 2, w.gaussian_peak)
    # reference constants: errormax 1e-3, nfmgmax 10
    rc, psi, g, st, _ = oracle_solve(h, rho, abi.default_params(abi.SFM_BC_PERIODIC))
    assert rc == abi.SFM_OK and st.converged == 1 and st.history()[-1] < 1e-3
    assert all(r >= 1e-3 for r in st.history()[:-1])
    # an unreachable tolerance ends on stagnation (ratio no longer halves) or nfmgmax
    rc, psi, g, st, _ = oracle_solve(h, rho, abi.default_params(abi.SFM_BC_PERIODIC, rel_tol=1e-30))
    assert rc == abi.SFM_ENOTCONVERGED and st.converged == 0
    hist = st.history()
    assert len(hist) == 10 or hist[-1] > 0.5 * hist[-2]


def test_zero_density_skips_the_loop():
    h = w.small_periodic(2, 8, 2, 0)
    rho = np.zeros((h.nblocks, 12, 12, 12))        # |resh2max| <= TINY: nfmgmax = 0 (fmg.F90:180)
    rc, psi, g, st, _ = oracle_solve(h, rho, abi.default_params(abi.SFM_BC_PERIODIC))
    assert rc == abi.SFM_OK and st.outer_iters == 0 and np.all(psi == 0.0)


def test_profile_accounts_for_the_solve_and_changes_nothing():
    """oracle_profile times each routine class exclusively: the classes add
    up to the whole solve, and the solve's results are those of oracle_solve."""
    from tests.oracle_lib import oracle_profile
    h = w.small_sphere(2, 8, 3, 2)
    p = abi.default_params(abi.SFM_BC_SPHERE, rel_tol=1e-10, max_outer=40, zero_mean=0)
    rho = w.block_field(h, p.ngh_io, w.softened_sphere)
    rc, secs, total, st = oracle_profile(h, rho, p)
    rc0, _, _, st0, _ = oracle_solve(h, rho, p)
    assert rc == rc0 == abi.SFM_OK
    assert st.outer_iters == st0.outer_iters and st.true_rel_residual == st0.true_rel_residual
    assert abs(sum(secs.values()) - total) <= 0.01 * total + 1e-4
    assert secs["ghost passes"] > 0 and secs["relaxation"] > 0 and secs["base grid"] > 0
