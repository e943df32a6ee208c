"""CUDA solver versus the CPU restatement (oracle) on the same seeded inputs.

FP64 path: the device kernels evaluate the reference's expressions in the
same order with --fmad=false (the multipole moments of the isolated boundary
included: one running sum per moment in the reference's cell order), so
every field must agree to the last bit, with the ghost cells filled by the
three directional passes or by one launch per level.  Mixed path: the FP32 inner solve
inside the FP64 defect correction must reach the same solution as the FP64
oracle to 1e-9 relative in phi (phi minus its mean for periodic boxes, whose
constant is free) and in g, at relative residual <= 1e-10.
"""
import ctypes as C

import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from code_only_b200.solver import FMGPoisson
from tests.oracle_lib import oracle_solve

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def interior(h, a, g):
    n = h.ni
    if a.ndim == 4:
        return a[:, g:g + n, g:g + n, g:g + n]
    return a[:, :, g:g + n, g:g + n, g:g + n]


CASES = {
    "uniform16_periodic": (lambda: w.uniform_periodic(2, 8), w.gaussian_peak, abi.SFM_BC_PERIODIC, {}),
    "amr2_periodic": (lambda: w.small_periodic(2, 8, 2, 0), w.gaussian_peak, abi.SFM_BC_PERIODIC, {}),
    "amr3_periodic": (lambda: w.small_periodic(2, 8, 3, 1), w.gaussian_peak, abi.SFM_BC_PERIODIC, {}),
    "amr3_periodic_ni16": (lambda: w.small_periodic(2, 16, 3, 4), w.gaussian_peak, abi.SFM_BC_PERIODIC, {}),
    "amr2_sphere": (lambda: w.small_sphere(2, 8, 2, 0), w.softened_sphere, abi.SFM_BC_SPHERE, {"zero_mean": 0}),
    "amr3_sphere_l4": (lambda: w.small_sphere(2, 8, 3, 2), w.softened_sphere, abi.SFM_BC_SPHERE,
                       {"zero_mean": 0, "lmax": 4}),
    "amr3_sphere_zeromean": (lambda: w.small_sphere(4, 8, 3, 3), w.softened_sphere, abi.SFM_BC_SPHERE, {}),
}


def force_ghost_fill(s, mode):
    """mode None: the tuning table (three passes by default); 1: one launch
    per level wherever that is exact; 0: always the three passes"""
    if mode is None:
        return
    lib = s.lib
    lib.sfm_debug_set_ghost_merge.argtypes = [C.c_void_p, C.c_int]
    lib.sfm_debug_set_ghost_merge.restype = C.c_int
    assert lib.sfm_debug_set_ghost_merge(s.ctx, mode) == abi.SFM_OK


@pytest.mark.parametrize("ghost", [None, 1], ids=["default", "one_launch_fill"])
@pytest.mark.parametrize("name", list(CASES))
def test_fp64_matches_oracle(name, ghost):
    mk, fn, bc, kw = CASES[name]
    h = mk()
    p = abi.default_params(bc, **kw)
    rho = w.block_field(h, p.ngh_io, fn)
    rc1, psi1, g1, st1, _ = oracle_solve(h, rho, p)
    with FMGPoisson(h, params=p) as s:
        force_ghost_fill(s, ghost)
        psi2, g2, st2 = s.solve(rho)
        # a second call on the same context must start from fresh arrays
        psi3, g3, st3 = s.solve(rho)
    assert rc1 == abi.SFM_OK and st1.outer_iters == st2.outer_iters
    tol = 0.0   # bit-identical: the isolated boundary's moments are summed in the reference's order too
    assert rel(interior(h, psi2, 2), interior(h, psi1, 2)) <= tol
    assert rel(psi2[:, 1:-1, 1:-1, 1:-1], psi1[:, 1:-1, 1:-1, 1:-1]) <= tol
    assert rel(interior(h, g2, 2), interior(h, g1, 2)) <= tol
    for a, b in zip(st1.history(), st2.history()):
        assert abs(a - b) <= tol * abs(a) + 1e-300
    assert np.array_equal(psi2, psi3) and np.array_equal(g2, g3)


@pytest.mark.parametrize("stage", [1, 2, 3, 4])
def test_fp64_stages_match_oracle(stage):
    h = w.small_periodic(2, 8, 3, 5)
    p = abi.default_params(abi.SFM_BC_PERIODIC)
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    _, _, _, _, d1 = oracle_solve(h, rho, p, stage=stage)
    lib = abi.load_library()
    lib.sfm_debug_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(abi.SfmStats),
                                    C.c_int, C.c_void_p]
    with FMGPoisson(h, params=p) as s:
        d2 = np.zeros_like(d1)
        psi = np.zeros_like(rho)
        rc = lib.sfm_debug_solve(s.ctx, rho.ctypes.data, psi.ctypes.data, None, None, stage, d2.ctypes.data)
        assert rc == 0
    assert np.array_equal(d1, d2)


def test_warm_start_matches_oracle():
    h = w.small_periodic(2, 8, 3, 6)
    p = abi.default_params(abi.SFM_BC_PERIODIC)
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    psi0 = w.block_field(h, p.ngh_io, lambda x, y, z: 0.1 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * z))
    rc1, psi1, g1, st1, _ = oracle_solve(h, rho, p, psi=psi0)
    with FMGPoisson(h, params=p) as s:
        psi2, g2, st2 = s.solve(rho, psi0)
    assert rel(psi2, psi1) == 0.0 and rel(interior(h, g2, 2), interior(h, g1, 2)) == 0.0


@pytest.mark.parametrize("ghost", [None, 1], ids=["default", "one_launch_fill"])
@pytest.mark.parametrize("name", ["amr3_periodic", "amr3_sphere_l4", "amr3_periodic_ni16"])
def test_mixed_precision_reaches_fp64_solution(name, ghost):
    mk, fn, bc, kw = CASES[name]
    h = mk()
    p64 = abi.default_params(bc, rel_tol=1e-10, max_outer=40, **kw)
    pmx = abi.default_params(bc, rel_tol=1e-10, max_outer=40, precision=abi.SFM_PREC_MIXED, **kw)
    rho = w.block_field(h, p64.ngh_io, fn)
    _, psi1, g1, st1, _ = oracle_solve(h, rho, p64)
    with FMGPoisson(h, params=pmx) as s:
        force_ghost_fill(s, ghost)
        psi2, g2, st2 = s.solve(rho)
    assert st2.true_rel_residual <= 1e-10
    a, b = interior(h, psi2, 2), interior(h, psi1, 2)
    if bc == abi.SFM_BC_PERIODIC:
        a, b = a - a.mean(), b - b.mean()
    assert rel(a, b) <= 1e-9
    assert rel(interior(h, g2, 2), interior(h, g1, 2)) <= 1e-9


def test_nonfinite_density_is_an_error():
    h = w.small_periodic(2, 8, 2, 0)
    p = abi.default_params(abi.SFM_BC_PERIODIC)
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    rho[3, 4, 4, 4] = np.nan
    with FMGPoisson(h, params=p) as s:
        st = abi.SfmStats()
        psi = np.zeros_like(rho)
        rc = s.lib.sfm_solve(s.ctx, rho.ctypes.data, psi.ctypes.data, None, C.byref(st))
    assert rc == abi.SFM_ENONFINITE


def test_host_g_writes_interiors_only():
    """sfm_solve stages g compact on the device and scatters the interiors into
    the caller's array: every io ghost entry keeps the caller's value, and the
    interiors equal those of the device-array entry point (full layout)."""
    import torch
    h = w.small_periodic(2, 8, 3, 1)
    p = abi.default_params(abi.SFM_BC_PERIODIC)
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    with FMGPoisson(h, params=p) as s:
        G = s.G
        sentinel = 12345.0
        g_host = np.full((h.nblocks, 3, G, G, G), sentinel)
        psi = np.zeros_like(rho)
        rc = s.lib.sfm_solve(s.ctx, rho.ctypes.data, psi.ctypes.data, g_host.ctypes.data, None)
        assert rc == abi.SFM_OK
        rho_d = torch.from_numpy(rho).cuda()
        psi_d = torch.zeros_like(rho_d)
        g_d = torch.full((h.nblocks, 3, G, G, G), -1.0, dtype=torch.float64, device="cuda")
        s.solve_device(rho_d.data_ptr(), psi_d.data_ptr(), g_d.data_ptr())
        torch.cuda.synchronize()
        g_dev = g_d.cpu().numpy()
    n, gw = h.ni, p.ngh_io
    inner = np.zeros((G, G, G), dtype=bool)
    inner[gw:gw + n, gw:gw + n, gw:gw + n] = True
    assert np.all(g_host[:, :, ~inner] == sentinel)
    assert np.array_equal(g_host[:, :, inner], g_dev[:, :, inner])
    assert np.array_equal(psi, psi_d.cpu().numpy())


def test_host_arrays_move_only_the_solved_region():
    """sfm_solve reads rho and psi on (-1:ni)^3 and writes psi there: the
    outer io ghost layer of rho may hold anything (NaN here) and psi's keeps
    the caller's values; the result equals the device-array call's, and the
    call reports the bytes it moved ((ni+2)^3 values per block for rho and
    psi each way, g's interiors out)."""
    import torch
    h = w.small_periodic(2, 8, 3, 1)
    p = abi.default_params(abi.SFM_BC_PERIODIC)
    assert p.ngh_io == 2
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    G, n = rho.shape[1], h.ni
    inner = np.zeros((G, G, G), dtype=bool)
    inner[1:G - 1, 1:G - 1, 1:G - 1] = True          # (-1:ni)^3
    rho_h = rho.copy()
    rho_h[:, ~inner] = np.nan
    psi_h = np.zeros_like(rho)
    psi_h[:, ~inner] = 777.0
    with FMGPoisson(h, params=p) as s:
        st = abi.SfmStats()
        rc = s.lib.sfm_solve(s.ctx, rho_h.ctypes.data, psi_h.ctypes.data, None, C.byref(st))
        assert rc == abi.SFM_OK
        rho_d = torch.from_numpy(rho).cuda()
        psi_d = torch.zeros_like(rho_d)
        s.solve_device(rho_d.data_ptr(), psi_d.data_ptr(), None)
        torch.cuda.synchronize()
        psi_dev = psi_d.cpu().numpy()
    assert np.all(psi_h[:, ~inner] == 777.0)
    assert np.array_equal(psi_h[:, inner], psi_dev[:, inner])
    staged = h.nblocks * (n + 2) ** 3 * 8
    assert st.h2d_bytes == 2 * staged and st.d2h_bytes == staged


def test_solve_device_rejects_host_pointers():
    """sfm_solve_device checks that every array is device memory of the
    context's device before it launches anything, and leaves the caller's
    current device as it found it."""
    import torch
    h = w.small_periodic(2, 8, 2, 0)
    p = abi.default_params(abi.SFM_BC_PERIODIC)
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    with FMGPoisson(h, params=p) as s:
        rho_d = torch.from_numpy(rho).cuda()
        psi_d = torch.zeros_like(rho_d)
        psi_h = np.zeros_like(rho)
        dev = torch.cuda.current_device()
        rc = s.lib.sfm_solve_device(s.ctx, C.c_void_p(rho.ctypes.data), C.c_void_p(psi_d.data_ptr()), None, None,
                                    None)
        assert rc == abi.SFM_EINVAL
        rc = s.lib.sfm_solve_device(s.ctx, C.c_void_p(rho_d.data_ptr()), C.c_void_p(psi_h.ctypes.data), None,
                                    None, None)
        assert rc == abi.SFM_EINVAL
        st = s.solve_device(rho_d.data_ptr(), psi_d.data_ptr())
        torch.cuda.synchronize()
        assert st.outer_iters > 0 and torch.cuda.current_device() == dev


def test_bounded_smoother_wait_reports_timeout():
    """Every mbarrier wait of the bulk-copy smoother is bounded.  With the
    consumers' poll limit set to zero every stage wait gives up at once: the
    CTA drains the copies it issued (their own wait keeps its full limit),
    sets the error flag and leaves, and the solve returns SFM_ETIMEOUT instead
    of hanging.  A fresh context afterwards solves bit-identically to the
    oracle, so the give-up left the GPU and the library usable."""
    lib = abi.load_library()
    lib.sfm_debug_set_wait_polls.argtypes = [C.c_void_p, C.c_uint32]
    lib.sfm_debug_set_wait_polls.restype = C.c_int
    h = w.small_periodic(2, 8, 2, 0)
    p = abi.default_params(abi.SFM_BC_PERIODIC, max_outer=1)
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    with FMGPoisson(h, params=p) as s:
        assert lib.sfm_debug_set_wait_polls(s.ctx, 0) == abi.SFM_OK
        psi = np.zeros_like(rho)
        rc = lib.sfm_solve(s.ctx, rho.ctypes.data, psi.ctypes.data, None, None)
        assert rc == abi.SFM_ETIMEOUT
    p = abi.default_params(abi.SFM_BC_PERIODIC)
    rc1, psi1, g1, st1, _ = oracle_solve(h, rho, p)
    with FMGPoisson(h, params=p) as s:
        psi2, g2, st2 = s.solve(rho)
    assert rel(psi2, psi1) == 0.0 and rel(interior(h, g2, 2), interior(h, g1, 2)) == 0.0


def test_bounded_wait_of_the_fused_sweep_reports_timeout():
    """The same give-up in the fused sweep of the mixed path (both colours
    per launch, one barrier of the consumer warps per tile): a warp whose
    stage wait failed still reaches the tile's barrier, the barrier's OR
    sends every consumer warp out, and the solve returns SFM_ETIMEOUT; the
    context then solves normally once the poll limit is restored."""
    lib = abi.load_library()
    lib.sfm_debug_set_wait_polls.argtypes = [C.c_void_p, C.c_uint32]
    lib.sfm_debug_set_wait_polls.restype = C.c_int
    h = w.small_periodic(2, 8, 2, 0)
    p = abi.default_params(abi.SFM_BC_PERIODIC, max_outer=1, precision=abi.SFM_PREC_MIXED)
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    with FMGPoisson(h, params=p) as s:
        s.load_tune_table(f"fused_sweeps 4 {h.ni} -1 -1 1\n")
        assert lib.sfm_debug_set_wait_polls(s.ctx, 0) == abi.SFM_OK
        psi = np.zeros_like(rho)
        rc = lib.sfm_solve(s.ctx, rho.ctypes.data, psi.ctypes.data, None, None)
        assert rc == abi.SFM_ETIMEOUT
    p = abi.default_params(abi.SFM_BC_PERIODIC, rel_tol=1e-10, max_outer=40, precision=abi.SFM_PREC_MIXED)
    with FMGPoisson(h, params=p) as s:
        s.load_tune_table(f"fused_sweeps 4 {h.ni} -1 -1 1\n")
        _, _, st = s.solve(rho)
    assert st.converged and st.true_rel_residual <= 1e-10


@pytest.mark.parametrize("name", ["amr3_periodic", "amr3_sphere_l4", "amr3_periodic_ni16"])
def test_red_black_sweeps_have_no_intra_colour_race(name):
    """Race check of the red-black smoother: with every colour sweep run one
    thread per block, the block's cells in the order of a serial sweep
    (sfm_debug_set_serial_relax), the solve must be bit-identical to the
    parallel kernels.  A cell of one colour that read another cell of the
    same colour while it was being updated would make the two differ."""
    mk, fn, bc, kw = CASES[name]
    h = mk()
    for prec in (abi.SFM_PREC_FP64, abi.SFM_PREC_MIXED):
        p = abi.default_params(bc, rel_tol=1e-10, max_outer=40, precision=prec, **kw)
        rho = w.block_field(h, p.ngh_io, fn)
        with FMGPoisson(h, params=p) as s:
            psi_par, g_par, st_par = s.solve(rho)
            s.lib.sfm_debug_set_serial_relax.argtypes = [C.c_void_p, C.c_int]
            s.lib.sfm_debug_set_serial_relax.restype = C.c_int
            assert s.lib.sfm_debug_set_serial_relax(s.ctx, 1) == abi.SFM_OK
            psi_ser, g_ser, st_ser = s.solve(rho)
        assert st_par.outer_iters == st_ser.outer_iters
        assert np.array_equal(psi_par, psi_ser) and np.array_equal(g_par, g_ser)


def test_solve_device_refuses_a_capturing_stream():
    """The solve synchronises with the host between outer iterations, so a
    stream under capture is refused before anything is queued on it, and the
    caller's capture stays valid."""
    import torch
    h = w.small_periodic(2, 8, 2, 0)
    p = abi.default_params(abi.SFM_BC_PERIODIC)
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    with FMGPoisson(h, params=p) as s:
        rho_d = torch.from_numpy(rho).cuda()
        psi_d = torch.zeros_like(rho_d)
        st = abi.SfmStats()
        stream = torch.cuda.Stream()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(stream):
            graph.capture_begin()
            rc = s.lib.sfm_solve_device(s.ctx, C.c_void_p(rho_d.data_ptr()), C.c_void_p(psi_d.data_ptr()), None,
                                        C.byref(st), C.c_void_p(stream.cuda_stream))
            psi_d.add_(1.0)   # the capture is still usable
            graph.capture_end()
        assert rc == abi.SFM_EINVAL
        graph.replay()
        torch.cuda.synchronize()
        assert float(psi_d.max()) == 1.0
        # and the same stream, not capturing, solves
        psi_d.zero_()
        rc = s.lib.sfm_solve_device(s.ctx, C.c_void_p(rho_d.data_ptr()), C.c_void_p(psi_d.data_ptr()), None,
                                    C.byref(st), C.c_void_p(stream.cuda_stream))
        torch.cuda.synchronize()
        assert rc == abi.SFM_OK
