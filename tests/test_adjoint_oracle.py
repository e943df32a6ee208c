"""The oracle's adjoint of the converged solve (CPU).

1. The transposed residual pipeline is the exact transpose of the forward
   one: <L phi, y> over leaf interiors equals <phi, L^T y> over every cell
   (physical ghosts included), to roundoff (1e-12 relative).
2. dJ/drho agrees with central finite differences of J(phi(rho)) for a
   linear J (weights on 16 seeded leaf cells).  The solve is linear in rho,
   so the central difference [J(rho + e) - J(rho - e)] / 2e equals J of the
   solve with a unit source at that cell; that is how it is evaluated here
   (the direct difference of two 1e-13 solves would lose the answer to
   cancellation).  Tolerance 1e-9 of the largest sampled sensitivity.
3. On a uniform periodic grid the operator is symmetric, so the adjoint is
   the forward solve run with the adjoint right-hand side.
"""
import ctypes as C

import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from tests.oracle_lib import leaf_mask, load_oracle, oracle_adjoint, oracle_solve

CASES = {
    "sphere_l3_lmax4": (lambda: w.small_sphere(2, 8, 3, 2), abi.SFM_BC_SPHERE, {"zero_mean": 0, "lmax": 4}),
    "sphere_l2_zero_mean": (lambda: w.small_sphere(2, 8, 2, 0), abi.SFM_BC_SPHERE, {}),
    "periodic_l3": (lambda: w.small_periodic(2, 8, 3, 1), abi.SFM_BC_PERIODIC, {}),
}


@pytest.mark.parametrize("name", list(CASES))
def test_transposed_pipeline_dot_product(name):
    mk, bc, kw = CASES[name]
    h = mk()
    lib = load_oracle()
    d = abi.HierDesc(h)
    p = abi.default_params(bc, **kw)
    rng = np.random.default_rng(11)
    lm = leaf_mask(h, 1)
    phi = rng.standard_normal(lm.shape)
    y = rng.standard_normal(lm.shape) * lm
    Lphi = np.zeros_like(phi)
    LTy = np.zeros_like(phi)
    assert lib.oracle_apply_L(d.ref(), C.byref(p), phi.ctypes.data, Lphi.ctypes.data) == abi.SFM_OK
    assert lib.oracle_apply_LT(d.ref(), C.byref(p), y.ctypes.data, LTy.ctypes.data) == abi.SFM_OK
    a = float((Lphi * y)[lm].sum())
    b = float((phi * LTy).sum())
    assert abs(a - b) <= 1e-12 * abs(a)


def _functional(h, gw, rng, periodic):
    lm = leaf_mask(h, gw)
    cells = np.argwhere(lm)
    pick = cells[rng.choice(len(cells), 16, replace=False)]
    wts = rng.standard_normal(16)
    if periodic:
        wts -= wts.mean()        # phi's constant is free in a periodic box
    dJ = np.zeros(lm.shape)
    for (b, k, j, i), v in zip(pick, wts):
        dJ[b, k, j, i] += v
    return dJ, cells


@pytest.mark.parametrize("name", ["sphere_l3_lmax4", "periodic_l3"])
def test_adjoint_matches_central_differences(name):
    mk, bc, kw = CASES[name]
    h = mk()
    p = abi.default_params(bc, rel_tol=1e-13, max_outer=60, **kw)
    p.stagnation_exit = 0
    gw = p.ngh_io
    rng = np.random.default_rng(5)
    dJ, cells = _functional(h, gw, rng, bc == abi.SFM_BC_PERIODIC)
    rc, grad, st = oracle_adjoint(h, dJ, p)
    assert rc == abi.SFM_OK and st.true_rel_residual <= 1e-12
    fds, ads = [], []
    for b, k, j, i in cells[rng.choice(len(cells), 24, replace=False)]:
        unit = np.zeros_like(dJ)
        unit[b, k, j, i] = 1.0
        rc1, psi, _, _, _ = oracle_solve(h, unit, p, want_g=False)
        fd = float((dJ * psi).sum())
        if fd == 0.0:            # masked cell (outside the isolated sphere): no influence
            assert grad[b, k, j, i] == 0.0
            continue
        fds.append(fd)
        ads.append(grad[b, k, j, i])
    fds, ads = np.array(fds), np.array(ads)
    assert len(fds) >= 12
    # 1e-9 of the largest sampled sensitivity (cells far from every weight
    # have sensitivities orders of magnitude smaller)
    assert np.abs(ads - fds).max() <= 1e-9 * np.abs(fds).max()
    # nothing on covered blocks or ghost entries
    assert not np.any(grad[~leaf_mask(h, gw)])


def test_adjoint_equals_forward_solve_on_symmetric_grid():
    h = w.uniform_periodic(2, 8)
    p = abi.default_params(abi.SFM_BC_PERIODIC, rel_tol=1e-13, max_outer=60)
    p.stagnation_exit = 0
    gw = p.ngh_io
    rng = np.random.default_rng(9)
    lm = leaf_mask(h, gw)
    dJ = rng.standard_normal(lm.shape) * lm
    dJ[lm] -= dJ[lm].mean()
    rc, grad, _ = oracle_adjoint(h, dJ, p)
    assert rc == abi.SFM_OK
    rc2, phi, _, _, _ = oracle_solve(h, dJ, p, want_g=False)   # forward solve, adjoint right-hand side
    assert rc2 == abi.SFM_OK
    a = grad[lm] - grad[lm].mean()
    b = phi[lm] - phi[lm].mean()
    assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()
