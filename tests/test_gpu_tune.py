"""The autotuner on the GPU: every launch-shape candidate evaluates the same
expressions in the same order, so a tuned solve must be bit-identical to the
untuned one (and, in FP64, to the oracle); the table survives a save/load
round trip and an empty table restores the defaults."""
import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from code_only_b200.solver import FMGPoisson, SFMError
from tests.oracle_lib import oracle_solve

pytestmark = pytest.mark.gpu

CASES = {
    "amr3_periodic": (lambda: w.small_periodic(2, 8, 3, 1), w.gaussian_peak, abi.SFM_BC_PERIODIC, {}),
    "amr3_sphere_l4": (lambda: w.small_sphere(2, 8, 3, 2), w.softened_sphere, abi.SFM_BC_SPHERE,
                       {"zero_mean": 0, "lmax": 4}),
    "amr3_periodic_ni16": (lambda: w.small_periodic(2, 16, 3, 4), w.gaussian_peak, abi.SFM_BC_PERIODIC, {}),
}


@pytest.mark.parametrize("prec", [abi.SFM_PREC_FP64, abi.SFM_PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", list(CASES))
def test_tuned_solve_is_bitwise_unchanged(name, prec):
    mk, fn, bc, kw = CASES[name]
    h = mk()
    p = abi.default_params(bc, rel_tol=1e-10, max_outer=40, precision=prec, **kw)
    rho = w.block_field(h, p.ngh_io, fn)
    with FMGPoisson(h, params=p) as s:
        psi0, g0, st0 = s.solve(rho)
        s.autotune(2)
        table = s.tune_table()
        assert any(ln.startswith(("ghost_fill", "relax_threads", "resid_bpc")) for ln in table.splitlines())
        psi1, g1, st1 = s.solve(rho)
        s.load_tune_table("")
        assert s.tune_table().strip().splitlines()[1:] == []
        s.load_tune_table(table)
        assert s.tune_table() == table
        psi2, g2, st2 = s.solve(rho)
        with pytest.raises(SFMError):
            s.load_tune_table("relax_threads 4 8 -1 -1 100\n")
        assert s.tune_table() == table            # a rejected table leaves the old one
    assert np.array_equal(psi0, psi1) and np.array_equal(g0, g1)
    assert np.array_equal(psi0, psi2) and np.array_equal(g0, g2)
    assert st0.outer_iters == st1.outer_iters
    if prec == abi.SFM_PREC_FP64:
        _, psi_o, g_o, _, _ = oracle_solve(h, rho, abi.default_params(bc, rel_tol=1e-10, max_outer=40, **kw))
        assert np.array_equal(psi1[:, 1:-1, 1:-1, 1:-1], psi_o[:, 1:-1, 1:-1, 1:-1])


@pytest.mark.parametrize("name", list(CASES))
def test_tuned_mixed_schedule_keeps_the_fp64_solution(name):
    """With a density, sfm_autotune also tunes the schedule of the mixed
    path's FP32 inner solve (V-cycles, sweeps, base-grid corrections).  The
    FP64 defect correction still converges to the same potential: within
    1e-9 (max norm, relative; phi's mean removed on periodic boxes) of the
    FP64 oracle in phi and g, at relative residual <= 1e-10."""
    import torch
    mk, fn, bc, kw = CASES[name]
    h = mk()
    p = abi.default_params(bc, rel_tol=1e-10, max_outer=40, precision=abi.SFM_PREC_MIXED, **kw)
    rho = w.block_field(h, p.ngh_io, fn)
    rho_d = torch.from_numpy(rho).cuda()
    with FMGPoisson(h, params=p) as s:
        s.autotune(2, rho_d.data_ptr())
        table = s.tune_table()
        for knob in ("fmg_ncycle", "fmg_sweeps", "vmg_sweeps", "base_corrections", "fused_sweeps", "local_sweeps"):
            assert any(ln.startswith(knob + " 4 ") for ln in table.splitlines()), knob
        psi2, g2, st2 = s.solve(rho)
    assert st2.converged and st2.true_rel_residual <= 1e-10
    _, psi1, g1, _, _ = oracle_solve(h, rho, abi.default_params(bc, rel_tol=1e-10, max_outer=40, **kw))
    n = h.ni
    a, b = psi2[:, 2:2 + n, 2:2 + n, 2:2 + n], psi1[:, 2:2 + n, 2:2 + n, 2:2 + n]
    if bc == abi.SFM_BC_PERIODIC:
        a, b = a - a.mean(), b - b.mean()
    assert np.abs(a - b).max() / np.abs(b).max() <= 1e-9
    ga, gb = g2[:, :, 2:2 + n, 2:2 + n, 2:2 + n], g1[:, :, 2:2 + n, 2:2 + n, 2:2 + n]
    assert np.abs(ga - gb).max() / np.abs(gb).max() <= 1e-9


@pytest.mark.parametrize("mask,local", [(1, 1), (2, 1), (3, 1), (1, 2), (3, 2), (3, 3)])
@pytest.mark.parametrize("name", list(CASES))
def test_fused_sweep_keeps_the_fp64_solution(name, mask, local):
    """fused_sweeps bit 0 makes every smoothing sweep of the mixed path's
    FP32 fmg_lin one launch for both colours (the second colour with the
    ghost cells and reflux fluxes of before the sweep), bit 1 the same for
    the sweeps of vmg_fas; local_sweeps 2 runs two full sweeps on the staged
    block per launch.  The FP64 defect correction must still reach the
    FP64 oracle's potential within 1e-9 at relative residual <= 1e-10, the
    profiled launches must report two colours each, and a solve after the
    table is cleared runs the two-launch sweep again (one colour each)."""
    mk, fn, bc, kw = CASES[name]
    h = mk()
    p = abi.default_params(bc, rel_tol=1e-10, max_outer=40, precision=abi.SFM_PREC_MIXED, profile=1, **kw)
    rho = w.block_field(h, p.ngh_io, fn)
    with FMGPoisson(h, params=p) as s:
        s.load_tune_table(f"fused_sweeps 4 {h.ni} -1 -1 {mask}\nlocal_sweeps 4 {h.ni} -1 -1 {local}\n")
        psi2, g2, st2 = s.solve(rho)
        psi3, g3, _ = s.solve(rho)                     # the graph replayed
        s.load_tune_table("")
        _, _, st4 = s.solve(rho)
    assert st2.converged and st2.true_rel_residual <= 1e-10
    assert st2.smoother_colours == (2 * local if mask & 1 else 1) and st2.smoother_launches > 0
    assert st4.smoother_colours == 1
    assert np.array_equal(psi2, psi3) and np.array_equal(g2, g3)
    _, psi1, g1, _, _ = oracle_solve(h, rho, abi.default_params(bc, rel_tol=1e-10, max_outer=40, **kw))
    n = h.ni
    a, b = psi2[:, 2:2 + n, 2:2 + n, 2:2 + n], psi1[:, 2:2 + n, 2:2 + n, 2:2 + n]
    if bc == abi.SFM_BC_PERIODIC:
        a, b = a - a.mean(), b - b.mean()
    assert np.abs(a - b).max() / np.abs(b).max() <= 1e-9
    ga, gb = g2[:, :, 2:2 + n, 2:2 + n, 2:2 + n], g1[:, :, 2:2 + n, 2:2 + n, 2:2 + n]
    assert np.abs(ga - gb).max() / np.abs(gb).max() <= 1e-9


@pytest.mark.parametrize("nt", [288, 512, 544])
@pytest.mark.parametrize("name", ["amr3_periodic", "amr3_periodic_ni16"])
def test_smoother_cta_sizes_are_bitwise(name, nt):
    """Every CTA size of the bulk-copy smoother (warp 0 producing, 7, 8, 15
    or 16 consumer warps) computes each cell with the same expression: the
    FP64 solve stays bit-identical to the oracle, and the mixed solve with
    fused sweeps is bit-identical to the one with the default CTA size."""
    mk, fn, bc, kw = CASES[name]
    h = mk()
    edges = [e for e in (4, 8, 16) if e <= h.ni]
    p64 = abi.default_params(bc, rel_tol=1e-10, max_outer=40, **kw)
    rho = w.block_field(h, p64.ngh_io, fn)
    with FMGPoisson(h, params=p64) as s:
        s.load_tune_table("".join(f"relax_threads 8 {e} -1 -1 {nt}\n" for e in edges))
        psi, _, _ = s.solve(rho)
    _, psi_o, _, _, _ = oracle_solve(h, rho, p64)
    assert np.array_equal(psi[:, 1:-1, 1:-1, 1:-1], psi_o[:, 1:-1, 1:-1, 1:-1])
    pmx = abi.default_params(bc, rel_tol=1e-10, max_outer=40, precision=abi.SFM_PREC_MIXED, **kw)
    fused = f"fused_sweeps 4 {h.ni} -1 -1 3\n"
    with FMGPoisson(h, params=pmx) as s:
        s.load_tune_table(fused)
        psi_a, g_a, _ = s.solve(rho)
        s.load_tune_table(fused + "".join(f"relax_threads 4 {e} -1 {k} {nt}\n" for e in edges for k in (-1, 1)))
        psi_b, g_b, _ = s.solve(rho)
    assert np.array_equal(psi_a, psi_b) and np.array_equal(g_a, g_b)


def test_fused_sweep_is_ignored_in_fp64():
    """An FP64 context given fused_sweeps 1 still runs the reference's two
    colour launches and stays bit-identical to the oracle."""
    mk, fn, bc, kw = CASES["amr3_periodic"]
    h = mk()
    p = abi.default_params(bc, rel_tol=1e-10, max_outer=40, profile=1, **kw)
    rho = w.block_field(h, p.ngh_io, fn)
    with FMGPoisson(h, params=p) as s:
        s.load_tune_table(f"fused_sweeps 4 {h.ni} -1 -1 3\nfused_sweeps 8 {h.ni} -1 -1 3\n")
        psi2, _, st2 = s.solve(rho)
    assert st2.smoother_colours == 1
    _, psi1, _, _, _ = oracle_solve(h, rho, abi.default_params(bc, rel_tol=1e-10, max_outer=40, **kw))
    assert np.array_equal(psi2[:, 1:-1, 1:-1, 1:-1], psi1[:, 1:-1, 1:-1, 1:-1])


def test_fp64_context_keeps_the_reference_schedule():
    """The schedule knobs exist only for the mixed path: tuning an FP64
    context with a density adds none, and its solve stays bit-identical to
    the oracle."""
    import torch
    mk, fn, bc, kw = CASES["amr3_periodic"]
    h = mk()
    p = abi.default_params(bc, rel_tol=1e-10, max_outer=40, **kw)
    rho = w.block_field(h, p.ngh_io, fn)
    rho_d = torch.from_numpy(rho).cuda()
    with FMGPoisson(h, params=p) as s:
        s.autotune(2, rho_d.data_ptr())
        assert not any(ln.startswith(("fmg_ncycle", "fmg_sweeps", "vmg_sweeps", "base_corrections", "fused_sweeps",
                                      "local_sweeps"))
                       for ln in s.tune_table().splitlines())
        psi2, _, _ = s.solve(rho)
    _, psi1, _, _, _ = oracle_solve(h, rho, p)
    assert np.array_equal(psi2[:, 1:-1, 1:-1, 1:-1], psi1[:, 1:-1, 1:-1, 1:-1])


BASE_CASES = {
    "uniform128": (lambda: w.uniform_periodic(16, 8), 32),   # 32^3 base grid
    "amr_base16": (lambda: w.small_periodic(16, 8, 2, 3), 32),
    "uniform64": (lambda: w.uniform_periodic(8, 8), 16),     # 16^3 base grid
}


@pytest.mark.parametrize("nct,wide", [(2, 16), (4, 16), (8, 16), (8, 32), (16, 16), (4, 32)])
@pytest.mark.parametrize("name", list(BASE_CASES))
def test_base_grid_cluster_is_bitwise(name, nct, wide):
    """The base-grid multigrid as a cluster of CTAs (the large levels spread
    over every CTA, the small ones on CTA 0, the maxima over the cluster)
    computes every cell with the same expression: the FP64 solve stays
    bit-identical to the oracle whatever the shape.  A shape the GPU cannot
    hold resident falls back to one CTA, which must match as well."""
    mk, nbase = BASE_CASES[name]
    h = mk()
    p = abi.default_params(abi.SFM_BC_PERIODIC, rel_tol=1e-10, max_outer=30)
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    _, psi_o, g_o, st_o, _ = oracle_solve(h, rho, p)
    with FMGPoisson(h, params=p) as s:
        s.load_tune_table(f"base_ctas 8 {nbase} -1 -1 {nct}\nbase_wide 8 {nbase} -1 -1 {wide}\n")
        psi, g, st = s.solve(rho)
        psi2, g2, _ = s.solve(rho)                       # the graph replayed
    assert st.outer_iters == st_o.outer_iters
    assert np.array_equal(psi[:, 1:-1, 1:-1, 1:-1], psi_o[:, 1:-1, 1:-1, 1:-1])
    n = h.ni
    assert np.array_equal(g[:, :, 2:2 + n, 2:2 + n, 2:2 + n], g_o[:, :, 2:2 + n, 2:2 + n, 2:2 + n])
    assert np.array_equal(psi, psi2) and np.array_equal(g, g2)


def test_autotuned_base_grid_choice_is_recorded():
    mk, nbase = BASE_CASES["uniform128"]
    h = mk()
    p = abi.default_params(abi.SFM_BC_PERIODIC, rel_tol=1e-10, max_outer=30)
    with FMGPoisson(h, params=p) as s:
        s.autotune(2)
        lines = s.tune_table().splitlines()
    assert any(ln.startswith(f"base_ctas 8 {nbase} ") for ln in lines)
    assert any(ln.startswith(f"base_wide 8 {nbase} ") for ln in lines)
