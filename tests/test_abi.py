"""The C-ABI library builds, loads and exports every entry point declared in
include/*.h; argument checking works without a GPU (no compute calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from code_only_b200 import abi, workloads as w

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w[\w\s\*]*?\b(sfm_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported(sfmg_lib):
    names = declared_functions()
    assert set(abi.EXPORTED) <= set(names)
    for n in names:
        assert hasattr(sfmg_lib, n), n


def test_debug_hooks_are_exported(sfmg_lib):
    """The test hooks that tests/ binds by name (not part of include/sfmg.h)."""
    for n in ("sfm_debug_set_wait_polls", "sfm_debug_set_serial_relax", "sfm_debug_set_ghost_merge",
              "sfm_debug_solve", "sfm_debug_set_guard_bytes", "sfm_debug_check_guards"):
        assert hasattr(sfmg_lib, n), n
    sfmg_lib.sfm_debug_set_guard_bytes.argtypes = [C.c_uint64]
    assert sfmg_lib.sfm_debug_set_guard_bytes(1 << 31) == abi.SFM_EINVAL
    assert sfmg_lib.sfm_debug_set_guard_bytes(0) == abi.SFM_OK
    sfmg_lib.sfm_debug_check_guards.argtypes = [C.c_void_p, C.c_void_p]
    assert sfmg_lib.sfm_debug_check_guards(None, None) == abi.SFM_EINVAL


def test_link_blocks_argument_checks(sfmg_lib):
    """sfm_link_blocks rejects bad sizes before any device call, and reports
    a missing GPU rather than touching the pointers."""
    ngb = (C.c_int32 * 3)(2, 2, 2)
    per = (C.c_int32 * 3)(1, 1, 1)
    dummy = C.c_void_p(16)
    args = lambda nb, nlev, g: (nb, nlev, dummy, dummy, g, per, dummy, dummy, dummy, dummy, None)
    assert sfmg_lib.sfm_link_blocks(*args(0, 1, ngb)) == abi.SFM_EINVAL
    assert sfmg_lib.sfm_link_blocks(*args(8, 17, ngb)) == abi.SFM_EINVAL            # more than 16 levels
    big = (C.c_int32 * 3)(1 << 16, 2, 2)
    assert sfmg_lib.sfm_link_blocks(*args(8, 6, big)) == abi.SFM_EINVAL             # positions past 2^20
    assert sfmg_lib.sfm_link_blocks(8, 1, None, dummy, ngb, per, dummy, dummy, dummy, dummy, None) == abi.SFM_EINVAL
    import torch
    if not torch.cuda.is_available():
        assert sfmg_lib.sfm_link_blocks(*args(8, 1, ngb)) == abi.SFM_EDEVICE


def test_stats_record_is_one_json_line():
    import json
    st = abi.SfmStats()
    st.outer_iters, st.converged, st.elem_bytes = 3, 1, 4
    for i, v in enumerate((1e-2, 1e-4, 1e-6)):
        st.ratio[i] = v
    st.device_ms, st.smoother_ms, st.smoother_cells = 12.5, 2.0, 4000000
    h = w.small_periodic(2, 8, 2, 0)
    rec = st.record(h)
    assert rec["residual_history"] == [1e-2, 1e-4, 1e-6] and rec["precision"] == "mixed"
    assert rec["smoother"]["cell_updates_per_s"] == 2e9
    assert rec["hierarchy"]["blocks"] == h.nblocks and sum(rec["hierarchy"]["level_blocks"]) == h.nblocks
    line = json.dumps(rec)
    assert "\n" not in line and json.loads(line) == rec


def test_default_params_match_reference_constants(sfmg_lib):
    p = abi.SfmParams()
    sfmg_lib.sfm_default_params(C.byref(p))
    assert p.max_outer == 10 and p.rel_tol == 1e-3 and p.zero_mean == 1 and p.ngh_io == 2
    assert p.four_pi_G == 4.0 * np.pi and p.precision == abi.SFM_PREC_FP64


def test_strerror(sfmg_lib):
    for code in range(0, -10, -1):
        assert sfmg_lib.sfm_strerror(code)
    assert b"unknown" in sfmg_lib.sfm_strerror(-99)


def test_argument_errors(sfmg_lib):
    h = w.small_periodic(2, 8, 2, 0)
    ctx = C.c_void_p()
    p = abi.default_params()
    assert sfmg_lib.sfm_create(None, C.byref(p), C.byref(ctx)) == abi.SFM_EINVAL
    bad = abi.default_params(ngh_io=0)
    assert sfmg_lib.sfm_create(abi.HierDesc(h).ref(), C.byref(bad), C.byref(ctx)) == abi.SFM_EINVAL
    bad = abi.default_params(lmax=7)
    assert sfmg_lib.sfm_create(abi.HierDesc(h).ref(), C.byref(bad), C.byref(ctx)) == abi.SFM_EINVAL
    assert sfmg_lib.sfm_solve(None, None, None, None, None) == abi.SFM_EINVAL
    sfmg_lib.sfm_destroy(None)


def test_without_gpu_create_reports_no_device(sfmg_lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = w.small_periodic(2, 8, 2, 0)
    ctx = C.c_void_p()
    p = abi.default_params()
    assert sfmg_lib.sfm_create(abi.HierDesc(h).ref(), C.byref(p), C.byref(ctx)) == abi.SFM_EDEVICE


def test_noalloc_argument_checks_precede_device_work(sfmg_lib):
    """sizes and arguments are refused before any CUDA call; valid arguments
    without a GPU report SFM_EDEVICE (no kernel is launched on either path)"""
    f = sfmg_lib.sfm_uniform_solve_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                  C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_void_p]
    f.restype = C.c_int
    fake = 1 << 20                              # never dereferenced: every call below returns early
    ok = (1.0 / 32, 1.0, 1e-10, 10, None, None, None)
    assert f(fake, fake, abi.SFM_NOALLOC_MAX_N * 2, *ok) == abi.SFM_ESIZE
    assert f(fake, fake, 24, *ok) == abi.SFM_ESIZE
    assert f(fake, fake, 0, *ok) == abi.SFM_ESIZE
    assert f(None, fake, 32, *ok) == abi.SFM_EINVAL
    assert f(fake, fake, 32, 0.0, 1.0, 1e-10, 10, None, None, None) == abi.SFM_EINVAL
    assert f(fake, fake, 32, 1.0, 1.0, -1.0, 10, None, None, None) == abi.SFM_EINVAL
    assert f(fake, fake, 32, 1.0, 1.0, 1e-10, -1, None, None, None) == abi.SFM_EINVAL
    assert f(fake + 4, fake, 32, *ok) == abi.SFM_EINVAL
    try:
        import torch
        if torch.cuda.is_available():
            return
    except ImportError:
        pass
    assert f(fake, fake, 32, *ok) == abi.SFM_EDEVICE
