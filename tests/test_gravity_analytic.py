"""Gravity against an analytic field, per AMR level (the reference's gravity
test, main_grav_test.F90:49-134, eval_error_g).

An isolated Gaussian sphere rho = exp(-r^2 / (2 sigma^2)) at the centre of a
nested hierarchy (three concentric levels) has g = -G M(<r) r / r^3 with
M(<r) = (2 pi sigma^2)^(3/2) [erf(r / (sqrt(2) sigma)) - sqrt(2/pi) (r/sigma)
exp(-r^2 / (2 sigma^2))] (G = 1, 4 pi G = 4 pi).  Over the leaf cells of each
level the relative error |g - g_exact| / |g_exact| is reduced as the
reference reduces it: its maximum, sqrt(sum rel^2 / ncell) and
sum rel / ncell with ncell = cells per block x base blocks.  The solve must
be second-order accurate: every level's errors shrink about fourfold when
the blocks double their cells per edge (same hierarchy shape)."""
from math import erf, pi, sqrt

import numpy as np
import pytest

from code_only_b200 import abi, workloads as w

SIGMA = 0.05
_erf = np.vectorize(erf)


def rho_gauss(x, y, z):
    return np.exp(-(x * x + y * y + z * z) / (2 * SIGMA ** 2))


def g_exact(x, y, z):
    r = np.sqrt(x * x + y * y + z * z)
    m = (2 * pi * SIGMA ** 2) ** 1.5 * (_erf(r / (sqrt(2) * SIGMA))
                                         - np.sqrt(2 / pi) * (r / SIGMA) * np.exp(-r * r / (2 * SIGMA ** 2)))
    f = -m / r ** 3
    return f * x, f * y, f * z


def level_errors(h, g, gw):
    """{level: (max, L2, L1)} of the relative error of g on leaf interiors,
    normalised as eval_error_g does"""
    n = h.ni
    xs, ys, zs = w.cell_centres(h, 0)
    leaf = h.child[:, 0] < 0
    ncell = n ** 3 * int(np.prod(h.ngb))
    out = {}
    for L in range(h.nlev):
        bs = np.nonzero(leaf & (h.level == L))[0]
        ex, ey, ez = g_exact(xs[bs][:, None, None, :], ys[bs][:, None, :, None], zs[bs][:, :, None, None])
        gg = g[bs][:, :, gw:gw + n, gw:gw + n, gw:gw + n]
        rel = np.sqrt((gg[:, 0] - ex) ** 2 + (gg[:, 1] - ey) ** 2 + (gg[:, 2] - ez) ** 2) / np.sqrt(
            ex ** 2 + ey ** 2 + ez ** 2)
        out[L] = (float(rel.max()), float(np.sqrt((rel ** 2).sum() / ncell)), float(rel.sum() / ncell))
    return out


def _params(precision=abi.SFM_PREC_FP64):
    return abi.default_params(abi.SFM_BC_SPHERE, rel_tol=1e-10, max_outer=40, zero_mean=0, precision=precision)


def _check(errs):
    e8, e16 = errs
    for L in e8:
        assert e8[L][0] < 1.5e-2 and e8[L][1] < 5e-3, (L, e8[L])
        assert e16[L][0] < 4e-3 and e16[L][1] < 1.3e-3, (L, e16[L])
        for q in range(3):   # second order: about 4x per doubling
            assert e8[L][q] / e16[L][q] > 3.4, (L, q, e8[L][q], e16[L][q])


def test_oracle_gravity_is_second_order():
    from tests.oracle_lib import oracle_solve
    errs = []
    for ni in (8, 16):
        h = w.nested_sphere(3, 4, ni)
        p = _params()
        rc, _, g, st, _ = oracle_solve(h, w.block_field(h, p.ngh_io, rho_gauss), p)
        assert rc == abi.SFM_OK
        errs.append(level_errors(h, g, p.ngh_io))
    _check(errs)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.SFM_PREC_FP64, abi.SFM_PREC_MIXED], ids=["fp64", "mixed"])
def test_device_gravity_is_second_order(prec):
    from code_only_b200.solver import FMGPoisson
    errs = []
    for ni in (8, 16):
        h = w.nested_sphere(3, 4, ni)
        p = _params(prec)
        with FMGPoisson(h, params=p) as s:
            _, g, st = s.solve(w.block_field(h, p.ngh_io, rho_gauss))
        assert st.converged
        errs.append(level_errors(h, g, p.ngh_io))
    _check(errs)
