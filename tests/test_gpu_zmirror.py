"""The z-mirror boundary on the GPU (fmg_boundary_phys_zmirror.F90): the
mirror plane u(:,:,-1) = u(:,:,0) applied at every place the reference
calls fmg_boundary_u / vmg_boundary_u / mg_boundary_u, the mask radius
without -zmin and the moments' mirror factors.

FP64 must be bit-identical to the oracle (psi with its ghost layer, g, the
outer iteration count) on boxes whose base grid takes the reference's
base-level sweeps (3^3 base blocks) and boxes whose base grid runs the
serial multigrid with the mirror on its z-min face (2^3 and 8^3 base
blocks; on the latter also as a thread-block cluster).  The mixed path must
reach the FP64 oracle's potential within 1e-9, and the half box must give
the potential of the mirror-symmetric full box with the ordinary isolated
boundary."""
import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from code_only_b200.solver import FMGPoisson, SFMError
from tests.oracle_lib import oracle_solve

pytestmark = pytest.mark.gpu

CASES = {
    "base3_l3": lambda: w.mirror_sphere(3, 8, 3),
    "base2_l3": lambda: w.mirror_sphere(2, 8, 3),
    "base8_l2": lambda: w.mirror_sphere(8, 8, 2),
}


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def params(precision=abi.SFM_PREC_FP64, **kw):
    return abi.default_params(abi.SFM_BC_ZMIRROR, rel_tol=1e-10, max_outer=40, zero_mean=0,
                              precision=precision, **kw)


@pytest.fixture(scope="module")
def oracle_runs():
    out = {}
    for name, mk in CASES.items():
        h = mk()
        rho = w.block_field(h, 2, w.wide_sphere)
        out[name] = (h, rho, oracle_solve(h, rho, params()))
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_zmirror_fp64_bitwise(oracle_runs, name):
    h, rho, (rc, psi1, g1, st1, _) = oracle_runs[name]
    assert rc == abi.SFM_OK
    with FMGPoisson(h, params=params()) as s:
        psi2, g2, st2 = s.solve(rho)
    n = h.ni
    assert st2.outer_iters == st1.outer_iters
    assert np.array_equal(psi2[:, 1:-1, 1:-1, 1:-1], psi1[:, 1:-1, 1:-1, 1:-1])
    assert np.array_equal(g2[:, :, 2:2 + n, 2:2 + n, 2:2 + n], g1[:, :, 2:2 + n, 2:2 + n, 2:2 + n])


@pytest.mark.parametrize("nct", [4, 16])
def test_zmirror_base_grid_cluster_bitwise(oracle_runs, nct):
    """The 16^3 base grid of the 8^3-block box as a cluster: the mirror
    steps spread over every CTA on the large levels."""
    h, rho, (rc, psi1, g1, st1, _) = oracle_runs["base8_l2"]
    with FMGPoisson(h, params=params()) as s:
        s.load_tune_table(f"base_ctas 8 16 -1 -1 {nct}\nbase_wide 8 16 -1 -1 16\n")
        psi2, _, st2 = s.solve(rho)
    assert st2.outer_iters == st1.outer_iters
    assert np.array_equal(psi2[:, 1:-1, 1:-1, 1:-1], psi1[:, 1:-1, 1:-1, 1:-1])


@pytest.mark.parametrize("tuned", [False, True], ids=["reference_schedule", "tuned"])
@pytest.mark.parametrize("name", list(CASES))
def test_zmirror_mixed_within_1e9(oracle_runs, name, tuned):
    import torch
    h, rho, (_, psi1, g1, _, _) = oracle_runs[name]
    with FMGPoisson(h, params=params(abi.SFM_PREC_MIXED)) as s:
        if tuned:
            rho_d = torch.from_numpy(rho).cuda()
            s.autotune(2, rho_d.data_ptr())
            del rho_d
        psi2, g2, st2 = s.solve(rho)
    n = h.ni
    assert st2.converged and st2.true_rel_residual <= 1e-10
    assert rel(psi2[:, 2:2 + n, 2:2 + n, 2:2 + n], psi1[:, 2:2 + n, 2:2 + n, 2:2 + n]) <= 1e-9
    assert rel(g2[:, :, 2:2 + n, 2:2 + n, 2:2 + n], g1[:, :, 2:2 + n, 2:2 + n, 2:2 + n]) <= 1e-9


def test_zmirror_half_box_equals_full_box_on_device():
    hh = w.mirror_sphere(3, 8, 3)
    hf = w.mirror_sphere(3, 8, 3, full=True)
    up = np.where(hf.x0[:, 2] > 0)[0]
    key = {(int(hh.level[b]), *np.round(hh.x0[b], 9)): b for b in range(hh.nblocks)}
    idx = np.array([key[(int(hf.level[b]), *np.round(hf.x0[b], 9))] for b in up])
    res = {}
    for name, h, bc in (("half", hh, abi.SFM_BC_ZMIRROR), ("full", hf, abi.SFM_BC_SPHERE)):
        p = abi.default_params(bc, rel_tol=1e-11, max_outer=40, zero_mean=0)
        with FMGPoisson(h, params=p) as s:
            res[name] = s.solve(w.block_field(h, 2, w.wide_sphere))
    n = hh.ni
    a = res["half"][0][idx][:, 2:2 + n, 2:2 + n, 2:2 + n]
    b = res["full"][0][up][:, 2:2 + n, 2:2 + n, 2:2 + n]
    assert rel(a, b) <= 1e-10


def test_zmirror_adjoint_is_refused():
    h = w.mirror_sphere(2, 8, 2)
    rho = w.block_field(h, 2, w.wide_sphere)
    with FMGPoisson(h, params=params()) as s:
        s.solve(rho)
        with pytest.raises(SFMError):
            s.adjoint(np.ones_like(rho))


@pytest.mark.parametrize("prec", [abi.SFM_PREC_FP64, abi.SFM_PREC_MIXED], ids=["fp64", "mixed"])
def test_mhd_be_sphere_matches_oracle(prec):
    """fmg_boundary_phys_sphere_MHD_BE.F90: the sphere boundary with the
    source masked outside the cloud radius Rcloud (params.r_cloud)."""
    h = w.small_sphere(2, 8, 3, 2)
    kw = dict(rel_tol=1e-10, max_outer=30, zero_mean=0, r_cloud=0.2)
    rho = w.block_field(h, 2, w.softened_sphere)
    _, psi1, g1, st1, _ = oracle_solve(h, rho, abi.default_params(abi.SFM_BC_SPHERE_MHD_BE, **kw))
    with FMGPoisson(h, params=abi.default_params(abi.SFM_BC_SPHERE_MHD_BE, precision=prec, **kw)) as s:
        psi2, g2, st2 = s.solve(rho)
    n = h.ni
    if prec == abi.SFM_PREC_FP64:
        assert st2.outer_iters == st1.outer_iters
        assert np.array_equal(psi2[:, 1:-1, 1:-1, 1:-1], psi1[:, 1:-1, 1:-1, 1:-1])
        assert np.array_equal(g2[:, :, 2:2 + n, 2:2 + n, 2:2 + n], g1[:, :, 2:2 + n, 2:2 + n, 2:2 + n])
    else:
        assert st2.converged and st2.true_rel_residual <= 1e-10
        assert rel(psi2[:, 2:2 + n, 2:2 + n, 2:2 + n], psi1[:, 2:2 + n, 2:2 + n, 2:2 + n]) <= 1e-9
