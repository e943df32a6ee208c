"""The z-periodic cylinder boundaries on the GPU
(fmg_boundary_phys_cyl_zperiodic.F90, fmg_boundary_phys_mask_zperiodic.F90):
the hierarchy wraps in z, the x and y faces get a00 ln(r) from the masked
source, and the base grid's multigrid wraps its z faces before every
relaxation and residual (mg_poisson.F90:16,56).

FP64 must be bit-identical to the oracle (psi with its ghost layer, g, the
outer iteration count; a00 sums the base cells in the reference's order and
ln(r) comes from the host's libm, as in the oracle), with the base grid on
one CTA and as a cluster; the mixed path within 1e-9 of the FP64 oracle."""
import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from code_only_b200.solver import FMGPoisson, SFMError
from tests.oracle_lib import oracle_solve

pytestmark = pytest.mark.gpu

MASK = 4 * np.pi * 0.05
CASES = {
    "cyl_base2": (lambda: w.zperiodic_cylinder(2, 8, 3), abi.SFM_BC_CYL_ZPERIODIC, 0.0),
    "mask_base2": (lambda: w.zperiodic_cylinder(2, 8, 3), abi.SFM_BC_MASK_ZPERIODIC, MASK),
    "cyl_base8": (lambda: w.zperiodic_cylinder(8, 8, 2), abi.SFM_BC_CYL_ZPERIODIC, 0.0),
}


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def params(bc, mask, precision=abi.SFM_PREC_FP64):
    return abi.default_params(bc, rel_tol=1e-10, max_outer=40, zero_mean=0, rho_mask=mask, precision=precision)


@pytest.fixture(scope="module")
def oracle_runs():
    out = {}
    for name, (mk, bc, mask) in CASES.items():
        h = mk()
        rho = w.block_field(h, 2, w.beaded_line)
        out[name] = (h, rho, oracle_solve(h, rho, params(bc, mask)))
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_cylinder_fp64_bitwise(oracle_runs, name):
    _, bc, mask = CASES[name]
    h, rho, (rc, psi1, g1, st1, _) = oracle_runs[name]
    assert rc == abi.SFM_OK
    with FMGPoisson(h, params=params(bc, mask)) as s:
        psi2, g2, st2 = s.solve(rho)
    n = h.ni
    assert st2.outer_iters == st1.outer_iters
    assert np.array_equal(psi2[:, 1:-1, 1:-1, 1:-1], psi1[:, 1:-1, 1:-1, 1:-1])
    assert np.array_equal(g2[:, :, 2:2 + n, 2:2 + n, 2:2 + n], g1[:, :, 2:2 + n, 2:2 + n, 2:2 + n])


@pytest.mark.parametrize("nct", [4, 16])
def test_cylinder_base_grid_cluster_bitwise(oracle_runs, nct):
    _, bc, mask = CASES["cyl_base8"]
    h, rho, (rc, psi1, _, st1, _) = oracle_runs["cyl_base8"]
    with FMGPoisson(h, params=params(bc, mask)) as s:
        s.load_tune_table(f"base_ctas 8 16 -1 -1 {nct}\nbase_wide 8 16 -1 -1 16\n")
        psi2, _, st2 = s.solve(rho)
    assert st2.outer_iters == st1.outer_iters
    assert np.array_equal(psi2[:, 1:-1, 1:-1, 1:-1], psi1[:, 1:-1, 1:-1, 1:-1])


@pytest.mark.parametrize("tuned", [False, True], ids=["reference_schedule", "tuned"])
@pytest.mark.parametrize("name", list(CASES))
def test_cylinder_mixed_within_1e9(oracle_runs, name, tuned):
    import torch
    _, bc, mask = CASES[name]
    h, rho, (_, psi1, g1, _, _) = oracle_runs[name]
    with FMGPoisson(h, params=params(bc, mask, abi.SFM_PREC_MIXED)) as s:
        if tuned:
            rho_d = torch.from_numpy(rho).cuda()
            s.autotune(2, rho_d.data_ptr())
            del rho_d
        psi2, g2, st2 = s.solve(rho)
    n = h.ni
    assert st2.converged and st2.true_rel_residual <= 1e-10
    assert rel(psi2[:, 2:2 + n, 2:2 + n, 2:2 + n], psi1[:, 2:2 + n, 2:2 + n, 2:2 + n]) <= 1e-9
    assert rel(g2[:, :, 2:2 + n, 2:2 + n, 2:2 + n], g1[:, :, 2:2 + n, 2:2 + n, 2:2 + n]) <= 1e-9


def test_cylinder_adjoint_is_refused():
    h = w.zperiodic_cylinder(2, 8, 2)
    rho = w.block_field(h, 2, w.beaded_line)
    with FMGPoisson(h, params=params(abi.SFM_BC_CYL_ZPERIODIC, 0.0)) as s:
        s.solve(rho)
        with pytest.raises(SFMError):
            s.adjoint(np.ones_like(rho))
