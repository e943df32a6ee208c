"""Block sizes at the ends of the supported range (sfm_hier_desc.ni: powers of
two from 4 to 64), and base boxes that are neither cubic nor powers of two.
The benchmark hierarchies use 8^3 and 16^3 blocks, whose fmg levels run the
tiled and bulk-copy kernels; blocks of 4^3 have a single coarser fmg level,
and 32^3 and 64^3 blocks start on the per-cell functors before reaching the
tiled sizes.  FP64 must equal the oracle bit for bit, mixed precision stay
within 1e-9 of it (phi -- mean removed on periodic boxes -- and g)."""
import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from code_only_b200.solver import FMGPoisson
from tests.oracle_lib import oracle_solve

pytestmark = pytest.mark.gpu


def _corner_refined(ngb, periodic):
    """a box of ngb base blocks (not cubic, not powers of two: the base level
    is relaxed by vmg sweeps, vmg.F90:85-91,397-402) with one column refined"""
    return w.build_hierarchy(ngb, 8, 2, lambda L, q, g: (q[:, 0] == 0) & (q[:, 1] == 1), periodic,
                             box_lo=(0.0, 0.0, 0.0) if periodic else (-0.5, -0.5, -0.5), box_size=1.0)


# name: (hierarchy, boundary, density)
CASES = {
    "ni4_amr3": (lambda: w.small_periodic(2, 4, 3, 1), abi.SFM_BC_PERIODIC, w.gaussian_peak),
    "ni32_amr2": (lambda: w.small_periodic(2, 32, 2, 0), abi.SFM_BC_PERIODIC, w.gaussian_peak),
    "ni64_uniform": (lambda: w.uniform_periodic(2, 64), abi.SFM_BC_PERIODIC, w.gaussian_peak),
    "box_2x3x4_periodic": (lambda: _corner_refined((2, 3, 4), True), abi.SFM_BC_PERIODIC, w.gaussian_peak),
    "box_3x2x5_isolated": (lambda: _corner_refined((3, 2, 5), False), abi.SFM_BC_SPHERE, w.softened_sphere),
}


def _params(bc, prec=abi.SFM_PREC_FP64):
    kw = {} if bc == abi.SFM_BC_PERIODIC else {"zero_mean": 0}
    return abi.default_params(bc, rel_tol=1e-10, max_outer=40, precision=prec, **kw)


@pytest.fixture(scope="module")
def oracle_runs():
    out = {}
    for name, (mk, bc, fn) in CASES.items():
        h = mk()
        p = _params(bc)
        rho = w.block_field(h, p.ngh_io, fn)
        rc, psi, g, st, _ = oracle_solve(h, rho, p)
        assert rc == abi.SFM_OK
        out[name] = (h, rho, psi, g)
    return out


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("prec", [abi.SFM_PREC_FP64, abi.SFM_PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", list(CASES))
def test_block_size_parity(oracle_runs, name, prec):
    h, rho, psi_o, g_o = oracle_runs[name]
    bc = CASES[name][1]
    p = _params(bc, prec)
    with FMGPoisson(h, params=p) as s:
        psi, g, st = s.solve(rho)
    assert st.converged
    n, gw = h.ni, p.ngh_io
    inner = (slice(None), slice(gw, gw + n), slice(gw, gw + n), slice(gw, gw + n))
    if prec == abi.SFM_PREC_FP64:
        assert np.array_equal(psi[inner], psi_o[inner])
        assert np.array_equal(g[:, :, gw:gw + n, gw:gw + n, gw:gw + n], g_o[:, :, gw:gw + n, gw:gw + n, gw:gw + n])
    else:
        a, b = psi[inner], psi_o[inner]
        if bc == abi.SFM_BC_PERIODIC:   # a periodic box fixes phi up to a constant
            a, b = a - a.mean(), b - b.mean()
        assert _rel(a, b) <= 1e-9
        assert _rel(g[:, :, gw:gw + n, gw:gw + n, gw:gw + n], g_o[:, :, gw:gw + n, gw:gw + n, gw:gw + n]) <= 1e-9
