"""Adjoint of the converged solve on the GPU (sfm_adjoint).

1. Against the oracle's adjoint on small hierarchies, FP64 and mixed
   precision: 1e-9 of the largest gradient entry (the Krylov solve runs to a
   relative residual of 1e-12 on both sides; the GPU's transposed ghost pass
   accumulates with atomics, so agreement is to roundoff, not bitwise).
2. The nested isolated-sphere workload (5 levels, 2560 blocks, multipoles to
   l = 4): gradients of W = 1/2 sum(rho phi dV) and of phi sampled
   trilinearly at 16 seeded points inside finest-level blocks, checked by
   central finite differences at 64 seeded cells spread over all levels.
   The solve is linear in rho, so [J(rho + e) - J(rho - e)] / 2e is
   evaluated through a solve of the unit source at that cell (W is quadratic,
   so its central difference is exact as well); agreement to 1e-6 of the
   largest sampled derivative.
3. On a uniform periodic grid the operator is symmetric: the adjoint equals
   the forward solve run with the adjoint right-hand side.
"""
import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from code_only_b200.solver import FMGPoisson
from tests.oracle_lib import leaf_mask, oracle_adjoint

pytestmark = pytest.mark.gpu

SMALL = {
    "sphere_l3_lmax4": (lambda: w.small_sphere(2, 8, 3, 2), abi.SFM_BC_SPHERE, {"zero_mean": 0, "lmax": 4}),
    "sphere_l2_zero_mean": (lambda: w.small_sphere(2, 8, 2, 0), abi.SFM_BC_SPHERE, {}),
    "periodic_l3": (lambda: w.small_periodic(2, 8, 3, 1), abi.SFM_BC_PERIODIC, {}),
}


def _params(bc, precision, **kw):
    p = abi.default_params(bc, rel_tol=1e-12, max_outer=60, precision=precision, **kw)
    p.stagnation_exit = 0
    return p


@pytest.mark.parametrize("precision", [abi.SFM_PREC_FP64, abi.SFM_PREC_MIXED])
@pytest.mark.parametrize("name", list(SMALL))
def test_adjoint_matches_oracle(name, precision):
    mk, bc, kw = SMALL[name]
    h = mk()
    p = _params(bc, precision, **kw)
    lm = leaf_mask(h, p.ngh_io)
    rng = np.random.default_rng(3)
    dJ = rng.standard_normal(lm.shape)          # covered-block entries act through the restriction
    rc1, g1, st1 = oracle_adjoint(h, dJ, _params(bc, abi.SFM_PREC_FP64, **kw))
    assert rc1 == abi.SFM_OK
    with FMGPoisson(h, params=p) as s:
        g2, st2 = s.adjoint(dJ)
        g3, _ = s.adjoint(dJ)                   # a second call on the same context
    assert st2.true_rel_residual <= 1e-12
    scale = np.abs(g1).max()
    assert np.abs(g2 - g1).max() <= 1e-9 * scale
    assert np.abs(g3 - g1).max() <= 1e-9 * scale
    assert not np.any(g2[~lm])


def _cell_volumes(h, gw):
    dv = (np.asarray(h.cellwidth)[np.asarray(h.level)] ** 3)
    return np.broadcast_to(dv[:, None, None, None], (h.nblocks,) + (h.ni + 2 * gw,) * 3)


def _sinks(h, gw, rng, count=16):
    """dJ/dphi of the sum of phi at `count` uniform points inside finest-level
    blocks, trilinear in the cell-centred values; the points stay at least
    half a cell inside their block so that only interior cells carry weight"""
    n = h.ni
    fine = np.flatnonzero(np.asarray(h.level) == h.nlev - 1)
    dJ = np.zeros((h.nblocks,) + (n + 2 * gw,) * 3)
    for _ in range(count):
        b = int(rng.choice(fine))
        u = rng.uniform(0.0, n - 1, size=3)      # cell-centre coordinates along x, y, z
        i0 = np.minimum(np.floor(u).astype(int), n - 2)
        t = u - i0
        for c in range(8):
            o = [(c >> d) & 1 for d in range(3)]
            wgt = np.prod([t[d] if o[d] else 1.0 - t[d] for d in range(3)])
            dJ[b, gw + i0[2] + o[2], gw + i0[1] + o[1], gw + i0[0] + o[0]] += wgt
    return dJ


def test_config4_gradients_match_central_differences():
    h, fn, bc = w.config_hierarchy("nested5")
    p = _params(bc, abi.SFM_PREC_FP64, zero_mean=0, lmax=4)
    gw = p.ngh_io
    rho = w.block_field(h, gw, fn)
    lm = leaf_mask(h, gw)
    dv = _cell_volumes(h, gw)
    rng = np.random.default_rng(777)
    dJ2 = _sinks(h, gw, rng)
    with FMGPoisson(h, params=p) as s:
        phi, _, st = s.solve(rho, want_g=False)
        assert st.true_rel_residual <= 1e-11
        gW, stW = s.adjoint(0.5 * rho * dv * lm)
        gW = gW + 0.5 * phi * dv * lm             # W depends on rho explicitly as well
        g2, st2 = s.adjoint(dJ2)
        assert stW.true_rel_residual <= 1e-12 and st2.true_rel_residual <= 1e-12
        # 64 seeded cells spread over all levels (covered cells included)
        crng = np.random.default_rng(4242)
        fdW, fd2, adW, ad2 = [], [], [], []
        for _ in range(64):
            L = int(crng.integers(0, h.nlev))
            blocks = np.flatnonzero(np.asarray(h.level) == L)
            b = int(crng.choice(blocks))
            i, j, k = (int(v) + gw for v in crng.integers(0, h.ni, size=3))
            unit = np.zeros_like(rho)
            unit[b, k, j, i] = 1.0
            resp, _, _ = s.solve(unit, want_g=False)
            fdW.append(0.5 * (dv[b, k, j, i] * phi[b, k, j, i] * lm[b, k, j, i] + float((rho * dv * lm * resp).sum())))
            fd2.append(float((dJ2 * resp).sum()))
            adW.append(gW[b, k, j, i])
            ad2.append(g2[b, k, j, i])
    for fd, ad in ((np.array(fdW), np.array(adW)), (np.array(fd2), np.array(ad2))):
        assert np.abs(fd).max() > 0
        assert np.abs(ad - fd).max() <= 1e-6 * np.abs(fd).max()


def test_adjoint_equals_forward_solve_on_symmetric_grid():
    h = w.uniform_periodic(2, 8)
    p = _params(abi.SFM_BC_PERIODIC, abi.SFM_PREC_FP64)
    lm = leaf_mask(h, p.ngh_io)
    rng = np.random.default_rng(9)
    dJ = rng.standard_normal(lm.shape) * lm
    dJ[lm] -= dJ[lm].mean()
    with FMGPoisson(h, params=p) as s:
        grad, _ = s.adjoint(dJ)
        phi, _, _ = s.solve(dJ, want_g=False)   # forward solve, adjoint right-hand side
    a = grad[lm] - grad[lm].mean()
    b = phi[lm] - phi[lm].mean()
    assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()
