"""ctypes mirror of include/sfmg.h and the loader of the in-tree CUDA library.

The library is built in-tree (``code_only_b200/_lib/libsfmg.so``) by
``code_only_b200/build.py``; importing this module never compiles anything and
loading fails loudly if the library is missing -- there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsfmg.so")

SFM_OK = 0
SFM_EINVAL = -1
SFM_EHIER = -2
SFM_ECUDA = -3
SFM_ENOMEM = -4
SFM_ENOTCONVERGED = -5
SFM_ENONFINITE = -6
SFM_EDEVICE = -7
SFM_ETIMEOUT = -8
SFM_ESIZE = -9

SFM_BC_PERIODIC = 0
SFM_BC_SPHERE = 1
SFM_BC_ZMIRROR = 2
SFM_BC_CYL_ZPERIODIC = 3
SFM_BC_MASK_ZPERIODIC = 4
SFM_BC_SPHERE_MHD_BE = 5
SFM_PREC_FP64 = 0
SFM_PREC_MIXED = 1
SFM_MAX_HISTORY = 64

# every exported symbol of include/sfmg.h
EXPORTED = ("sfm_default_params", "sfm_create", "sfm_solve", "sfm_solve_device",
            "sfm_adjoint", "sfm_destroy", "sfm_strerror", "sfm_info", "sfm_autotune", "sfm_tune_save",
            "sfm_tune_load", "sfm_uniform_solve_noalloc", "sfm_link_blocks")
SFM_NOALLOC_MAX_N = 32


class SfmHierDesc(C.Structure):
    _fields_ = [
        ("nlev", C.c_int32), ("nblocks", C.c_int32),
        ("ni", C.c_int32), ("nj", C.c_int32), ("nk", C.c_int32),
        ("ngb", C.c_int32 * 3),
        ("level", C.POINTER(C.c_int32)), ("ijk", C.POINTER(C.c_int32)),
        ("parent", C.POINTER(C.c_int32)), ("child", C.POINTER(C.c_int32)),
        ("nbr", C.POINTER(C.c_int32)), ("touch", C.POINTER(C.c_int8)),
        ("cellwidth", C.POINTER(C.c_double)), ("x0", C.POINTER(C.c_double)),
    ]


class SfmParams(C.Structure):
    _fields_ = [
        ("bc", C.c_int32), ("lmax", C.c_int32), ("precision", C.c_int32),
        ("max_outer", C.c_int32), ("rel_tol", C.c_double), ("four_pi_G", C.c_double),
        ("zero_mean", C.c_int32), ("ngh_io", C.c_int32), ("report_residual", C.c_int32),
        ("stagnation_exit", C.c_int32), ("profile", C.c_int32), ("rho_mask", C.c_double),
        ("r_cloud", C.c_double),
    ]


class SfmStats(C.Structure):
    _fields_ = [
        ("outer_iters", C.c_int32), ("converged", C.c_int32), ("resh2max", C.c_double),
        ("ratio", C.c_double * SFM_MAX_HISTORY), ("true_rel_residual", C.c_double),
        ("rho_mean", C.c_double), ("device_ms", C.c_double), ("kernel_launches", C.c_int64),
        ("smoother_ms", C.c_double), ("smoother_launches", C.c_int64), ("smoother_cells", C.c_int64),
        ("elem_bytes", C.c_int32), ("smoother_colours", C.c_int32),
        ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64),
    ]

    def history(self):
        return [self.ratio[i] for i in range(min(self.outer_iters, SFM_MAX_HISTORY))]

    def record(self, hierarchy=None) -> dict:
        """The solve as one structured record (json.dumps gives one line): the
        outer residual history the reference prints once per iteration
        ('fmg error = ...', fmg.F90:189), the device time and launches, the
        smoother's share (filled when the context profiles), the bytes a
        host-array call moved, and the hierarchy's shape when given."""
        rec = {
            "outer_iters": int(self.outer_iters), "converged": bool(self.converged),
            "residual_history": self.history(), "true_rel_residual": float(self.true_rel_residual),
            "rho_mean": float(self.rho_mean), "precision": "fp64" if self.elem_bytes == 8 else "mixed",
            "device_ms": float(self.device_ms), "kernel_launches": int(self.kernel_launches),
            "smoother": {"ms": float(self.smoother_ms), "launches": int(self.smoother_launches),
                         "cell_updates": int(self.smoother_cells), "colours_per_launch": int(self.smoother_colours),
                         "cell_updates_per_s": (float(self.smoother_cells) / (self.smoother_ms * 1e-3)
                                                if self.smoother_ms > 0 else None)},
            "host_bytes": {"h2d": int(self.h2d_bytes), "d2h": int(self.d2h_bytes)},
        }
        if hierarchy is not None:
            rec["hierarchy"] = {"levels": int(hierarchy.nlev), "blocks": int(hierarchy.nblocks),
                                "block_cells": int(hierarchy.ni) ** 3,
                                "level_blocks": [int(v) for v in hierarchy.level_counts()]}
        return rec


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class HierDesc:
    """Keeps the numpy arrays of a Hierarchy alive behind an SfmHierDesc."""

    def __init__(self, h):
        h.contiguous()
        self.h = h
        d = SfmHierDesc()
        d.nlev = h.nlev
        d.nblocks = h.nblocks
        d.ni = d.nj = d.nk = h.ni
        for i in range(3):
            d.ngb[i] = h.ngb[i]
        self._keep = [h.level, h.ijk, h.parent, h.child, h.nbr, h.touch, h.cellwidth, h.x0]
        d.level = _ptr(h.level, C.c_int32)
        d.ijk = _ptr(h.ijk, C.c_int32)
        d.parent = _ptr(h.parent, C.c_int32)
        d.child = _ptr(h.child, C.c_int32)
        d.nbr = _ptr(h.nbr, C.c_int32)
        d.touch = _ptr(h.touch, C.c_int8)
        d.cellwidth = _ptr(h.cellwidth, C.c_double)
        d.x0 = _ptr(h.x0, C.c_double)
        self.desc = d

    def ref(self):
        return C.byref(self.desc)


def default_params(bc: int = SFM_BC_PERIODIC, **kw) -> SfmParams:
    """The reference's constants (fmg.F90:146,179; config.h:194), bc chosen."""
    p = SfmParams()
    p.bc = bc
    p.lmax = 3
    p.precision = SFM_PREC_FP64
    p.max_outer = 10
    p.rel_tol = 1e-3
    p.four_pi_G = 4.0 * np.pi
    p.zero_mean = 1
    p.ngh_io = 2
    p.report_residual = 1
    p.stagnation_exit = 1
    p.profile = 0
    p.rho_mask = 0.0
    p.r_cloud = 0.0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


_lib: Optional[C.CDLL] = None


def load_library(path: Optional[str] = None) -> C.CDLL:
    """Loads libsfmg.so; raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build the CUDA extension with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (no CPU fallback exists)")
    lib = C.CDLL(p)
    lib.sfm_default_params.argtypes = [C.POINTER(SfmParams)]
    lib.sfm_default_params.restype = None
    lib.sfm_create.argtypes = [C.POINTER(SfmHierDesc), C.POINTER(SfmParams), C.POINTER(C.c_void_p)]
    lib.sfm_create.restype = C.c_int
    lib.sfm_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(SfmStats)]
    lib.sfm_solve.restype = C.c_int
    lib.sfm_solve_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.POINTER(SfmStats), C.c_void_p]
    lib.sfm_solve_device.restype = C.c_int
    lib.sfm_adjoint.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(SfmStats)]
    lib.sfm_adjoint.restype = C.c_int
    lib.sfm_destroy.argtypes = [C.c_void_p]
    lib.sfm_destroy.restype = None
    lib.sfm_strerror.argtypes = [C.c_int]
    lib.sfm_strerror.restype = C.c_char_p
    lib.sfm_info.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    lib.sfm_info.restype = C.c_int
    lib.sfm_autotune.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    lib.sfm_autotune.restype = C.c_int
    lib.sfm_tune_save.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    lib.sfm_tune_save.restype = C.c_int
    lib.sfm_tune_load.argtypes = [C.c_void_p, C.c_char_p]
    lib.sfm_tune_load.restype = C.c_int
    lib.sfm_tune_text_check.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t]
    lib.sfm_tune_text_check.restype = C.c_int
    lib.sfm_link_blocks.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32),
                                    C.POINTER(C.c_int32), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]
    lib.sfm_link_blocks.restype = C.c_int
    if path is None:
        _lib = lib
    return lib
