"""Guard-band debug mode on the GPU (the library's bounds check).

With sfm_debug_set_guard_bytes, every device array of a new context sits
between two bands of 0xFF bytes.  A kernel that writes past either end of an
array changes a band (sfm_debug_check_guards counts the changed bytes); one
that reads past an end reads NaN (0xFF bytes are NaN in FP32 and FP64) and
the results change.  So: solves, the autotuner's launch-shape and schedule
candidates, and the adjoint run with bands around every array, the bands
must be intact afterwards, and the results must equal, bit for bit, those
of the same solve without bands (the adjoint, whose transposed ghost pass
adds into coarse cells with atomics, to roundoff).  No access is made to fault: a stray access
lands in a band, which is part of the allocation."""
import ctypes as C

import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from code_only_b200.solver import FMGPoisson

pytestmark = pytest.mark.gpu

GUARD = 64 * 1024

CASES = {
    "amr3_periodic": (lambda: w.small_periodic(2, 8, 3, 1), w.gaussian_peak, abi.SFM_BC_PERIODIC, {}),
    "amr3_sphere": (lambda: w.small_sphere(2, 8, 3, 2), w.softened_sphere, abi.SFM_BC_SPHERE, {"zero_mean": 0}),
    "amr3_periodic_ni16": (lambda: w.small_periodic(2, 16, 3, 4), w.gaussian_peak, abi.SFM_BC_PERIODIC, {}),
    "uniform64": (lambda: w.uniform_periodic(8, 8), w.gaussian_peak, abi.SFM_BC_PERIODIC, {}),
    "zmirror": (lambda: w.mirror_sphere(3, 8, 3), w.wide_sphere, abi.SFM_BC_ZMIRROR, {"zero_mean": 0}),
    "cyl_zperiodic": (lambda: w.zperiodic_cylinder(2, 8, 3), w.beaded_line, abi.SFM_BC_CYL_ZPERIODIC,
                      {"zero_mean": 0}),
}


def _hooks():
    lib = abi.load_library()
    lib.sfm_debug_set_guard_bytes.argtypes = [C.c_uint64]
    lib.sfm_debug_set_guard_bytes.restype = C.c_int
    lib.sfm_debug_check_guards.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    lib.sfm_debug_check_guards.restype = C.c_int
    return lib


def _bad_bytes(lib, s):
    bad = C.c_int64(-1)
    assert lib.sfm_debug_check_guards(s.ctx, C.byref(bad)) == abi.SFM_OK
    return bad.value


def _solve(h, p, rho, table, guard, lib, tune=False):
    assert lib.sfm_debug_set_guard_bytes(guard) == abi.SFM_OK
    try:
        with FMGPoisson(h, params=p) as s:
            if tune:
                import torch
                rho_d = torch.from_numpy(rho).cuda()
                s.autotune(1, rho_d.data_ptr())
                table = s.tune_table()
            elif table is not None:
                s.load_tune_table(table)
            psi, g, st = s.solve(rho)
            bad = _bad_bytes(lib, s) if guard else 0
    finally:
        lib.sfm_debug_set_guard_bytes(0)
    return psi, g, st, bad, table


@pytest.mark.parametrize("prec", [abi.SFM_PREC_FP64, abi.SFM_PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", list(CASES))
def test_guard_bands_stay_intact_and_results_unchanged(name, prec):
    lib = _hooks()
    mk, fn, bc, kw = CASES[name]
    h = mk()
    p = abi.default_params(bc, rel_tol=1e-10, max_outer=40, precision=prec, **kw)
    rho = w.block_field(h, p.ngh_io, fn)
    # the autotuner's candidates run inside the bands too; the table it
    # picks is then replayed without bands
    psi_g, g_g, st_g, bad, table = _solve(h, p, rho, None, GUARD, lib, tune=True)
    assert bad == 0, f"{bad} guard-band bytes changed"
    psi, g, st, _, _ = _solve(h, p, rho, table, 0, lib)
    assert st_g.outer_iters == st.outer_iters
    assert np.array_equal(psi_g, psi) and np.array_equal(g_g, g)
    assert np.isfinite(psi).all()


@pytest.mark.parametrize("name", ["amr3_periodic", "amr3_sphere"])
def test_guard_bands_around_the_adjoint(name):
    lib = _hooks()
    mk, fn, bc, kw = CASES[name]
    h = mk()
    p = abi.default_params(bc, rel_tol=1e-10, max_outer=40, precision=abi.SFM_PREC_MIXED, **kw)
    rho = w.block_field(h, p.ngh_io, fn)
    out = {}
    for guard in (GUARD, 0):
        assert lib.sfm_debug_set_guard_bytes(guard) == abi.SFM_OK
        try:
            with FMGPoisson(h, params=p) as s:
                psi, _, _ = s.solve(rho)
                lam, st = s.adjoint(psi, allow_unconverged=True)
                out[guard] = lam
                if guard:
                    assert _bad_bytes(lib, s) == 0
        finally:
            lib.sfm_debug_set_guard_bytes(0)
    # the transposed ghost pass scatters into coarse cells with FP64 atomics,
    # so the adjoint is reproducible to roundoff, not to the bit
    assert np.isfinite(out[GUARD]).all()
    assert np.abs(out[GUARD] - out[0]).max() <= 1e-9 * np.abs(out[0]).max()


def test_guard_setting_is_validated():
    lib = _hooks()
    assert lib.sfm_debug_set_guard_bytes(1 << 31) == abi.SFM_EINVAL
    assert lib.sfm_debug_set_guard_bytes(0) == abi.SFM_OK
