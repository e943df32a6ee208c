"""Python mirror of the reference's `fmg_poisson` entry point over the C ABI.

The reference's `fmg_poisson` (fmg.F90:63-74) takes no arguments: it reads the
hierarchy and the block arrays from module globals, solves
lap(phi) = 4 pi G (rho - <rho>) by FMG, and writes U(MPSI) (interior + 1
ghost layer) and U(MGX:MGZ) (interior) back.  Here the same data is passed
explicitly:

    ctx = FMGPoisson(hierarchy, bc=SFM_BC_SPHERE)        # fmg_data_init + fmg_alloc_LoL
    psi, g, stats = ctx.solve(rho, psi0)                 # fmg_cycle
    dJ_drho, astats = ctx.adjoint(dJ_dphi)               # adjoint (no reference counterpart)
    ctx.close()

``rho``/``psi0`` are float64 arrays [nblocks, G, G, G] (G = ni + 2*ngh_io,
i fastest in memory), as BlockMem(gid)%u(:,:,:,m) stores one component.
Errors raise SFMError carrying the library's status code; there is no CPU
path -- a missing or unloadable CUDA library raises.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import abi


class SFMError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        lib = abi.load_library()
        super().__init__(f"{what}: {lib.sfm_strerror(code).decode()} ({code})")


class FMGPoisson:
    def __init__(self, hierarchy, bc: int = abi.SFM_BC_PERIODIC, params: Optional[abi.SfmParams] = None, **kw):
        self.lib = abi.load_library()
        self.h = hierarchy
        self.desc = abi.HierDesc(hierarchy)
        self.params = params if params is not None else abi.default_params(bc, **kw)
        self.ctx = C.c_void_p()
        rc = self.lib.sfm_create(self.desc.ref(), C.byref(self.params), C.byref(self.ctx))
        if rc != abi.SFM_OK:
            self.ctx = None
            raise SFMError(rc, "sfm_create")
        self.G = hierarchy.ni + 2 * self.params.ngh_io

    @property
    def shape(self):
        return (self.h.nblocks, self.G, self.G, self.G)

    def solve(self, rho: np.ndarray, psi: Optional[np.ndarray] = None, want_g: bool = True, allow_unconverged=True):
        """One solve with host arrays (sfm_solve).  Returns (psi, g, stats)."""
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        if rho.shape != self.shape:
            raise ValueError(f"rho has shape {rho.shape}, expected {self.shape}")
        psi = np.zeros(self.shape) if psi is None else np.array(psi, dtype=np.float64, order="C", copy=True)
        g = np.zeros((self.h.nblocks, 3, self.G, self.G, self.G)) if want_g else None
        st = abi.SfmStats()
        rc = self.lib.sfm_solve(self.ctx, rho.ctypes.data, psi.ctypes.data,
                                g.ctypes.data if g is not None else None, C.byref(st))
        if rc not in (abi.SFM_OK, abi.SFM_ENOTCONVERGED) or (rc != abi.SFM_OK and not allow_unconverged):
            raise SFMError(rc, "sfm_solve")
        return psi, g, st

    def solve_device(self, rho_ptr: int, psi_ptr: int, g_ptr: Optional[int] = None, stream: int = 0):
        """Solve on device-resident buffers (sfm_solve_device); pointers as ints."""
        st = abi.SfmStats()
        rc = self.lib.sfm_solve_device(self.ctx, C.c_void_p(rho_ptr), C.c_void_p(psi_ptr),
                                       C.c_void_p(g_ptr) if g_ptr else None, C.byref(st),
                                       C.c_void_p(stream) if stream else None)
        if rc not in (abi.SFM_OK, abi.SFM_ENOTCONVERGED):
            raise SFMError(rc, "sfm_solve_device")
        return st

    def adjoint(self, dJ_dphi: np.ndarray, allow_unconverged=False):
        """Gradient of a functional of the converged potential (sfm_adjoint).

        dJ_dphi: [nblocks, G, G, G], dJ/dphi on block interiors (ghost entries
        ignored; entries on covered blocks act through the restriction that
        defines phi there).  Returns (dJ_drho, stats): dJ/drho on leaf
        interiors, zero elsewhere.  params.rel_tol is the tolerance on
        ||dJ/dphi - A^T lambda||_2 relative to ||dJ/dphi||_2 and
        params.max_outer the iteration cap of the Krylov solve."""
        dJ = np.ascontiguousarray(dJ_dphi, dtype=np.float64)
        if dJ.shape != self.shape:
            raise ValueError(f"dJ_dphi has shape {dJ.shape}, expected {self.shape}")
        out = np.zeros(self.shape)
        st = abi.SfmStats()
        rc = self.lib.sfm_adjoint(self.ctx, dJ.ctypes.data, out.ctypes.data, C.byref(st))
        if rc not in (abi.SFM_OK, abi.SFM_ENOTCONVERGED) or (rc != abi.SFM_OK and not allow_unconverged):
            raise SFMError(rc, "sfm_adjoint")
        return out, st

    def autotune(self, reps: int = 3, rho_ptr: Optional[int] = None):
        """Times every launch-shape candidate on this hierarchy and keeps the
        fastest (sfm_autotune; bit-identical results whatever is chosen).  With
        rho_ptr (device array of the density, sfm_solve_device's layout) a
        mixed-precision context also tunes its inner-solve schedule by complete
        solves of that density."""
        rc = self.lib.sfm_autotune(self.ctx, reps, C.c_void_p(rho_ptr) if rho_ptr else None)
        if rc != abi.SFM_OK:
            raise SFMError(rc, "sfm_autotune")

    def tune_table(self) -> str:
        """The tuning table as text (sfm_tune_save)."""
        n = C.c_size_t()
        rc = self.lib.sfm_tune_save(self.ctx, None, 0, C.byref(n))
        if rc != abi.SFM_OK:
            raise SFMError(rc, "sfm_tune_save")
        buf = C.create_string_buffer(n.value + 1)
        rc = self.lib.sfm_tune_save(self.ctx, buf, n.value + 1, None)
        if rc != abi.SFM_OK:
            raise SFMError(rc, "sfm_tune_save")
        return buf.value.decode()

    def load_tune_table(self, text: str):
        """Replaces the tuning table (sfm_tune_load); '' restores the defaults."""
        rc = self.lib.sfm_tune_load(self.ctx, text.encode())
        if rc != abi.SFM_OK:
            raise SFMError(rc, "sfm_tune_load")

    def info(self):
        lv = C.c_int32()
        by = C.c_int64()
        self.lib.sfm_info(self.ctx, C.byref(lv), C.byref(by))
        return {"fmg_levels": lv.value, "device_bytes": by.value}

    def close(self):
        if self.ctx:
            self.lib.sfm_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fmg_poisson(hierarchy, rho: np.ndarray, psi: np.ndarray, bc: int = abi.SFM_BC_PERIODIC, **kw):
    """One-shot form of the reference entry point: returns (psi, g, stats)."""
    with FMGPoisson(hierarchy, bc=bc, **kw) as s:
        return s.solve(rho, psi)


def link_blocks(level, ijk, ngb, periodic, nlev: Optional[int] = None, stream: int = 0):
    """Links of a block hierarchy computed on the device (sfm_link_blocks):
    the parent, children, same-level face neighbours and physical-boundary
    flags that the reference's refinement keeps (grid.F90:587-731), from the
    blocks' AMR levels and integer positions.

    level: int32 [nb], ijk: int32 [nb, 3] -- CUDA tensors of the current
    device; ngb: base blocks per direction; periodic: one bool or three.
    Returns (parent [nb], child [nb, 8], nbr [nb, 6], touch [nb, 6]) as CUDA
    tensors in sfm_hier_desc's conventions."""
    import torch
    nb = int(level.shape[0])
    if ijk.shape != (nb, 3) or level.dtype != torch.int32 or ijk.dtype != torch.int32:
        raise ValueError("level must be int32 [nb] and ijk int32 [nb, 3]")
    level, ijk = level.contiguous(), ijk.contiguous()
    if nlev is None:
        nlev = int(level.max().item()) + 1 if nb else 0
    per = (bool(periodic),) * 3 if np.isscalar(periodic) else tuple(bool(v) for v in periodic)
    dev = level.device
    parent = torch.empty(nb, dtype=torch.int32, device=dev)
    child = torch.empty((nb, 8), dtype=torch.int32, device=dev)
    nbr = torch.empty((nb, 6), dtype=torch.int32, device=dev)
    touch = torch.empty((nb, 6), dtype=torch.int8, device=dev)
    lib = abi.load_library()
    rc = lib.sfm_link_blocks(nb, int(nlev), level.data_ptr(), ijk.data_ptr(), (C.c_int32 * 3)(*[int(v) for v in ngb]),
                             (C.c_int32 * 3)(*[int(v) for v in per]), parent.data_ptr(), child.data_ptr(),
                             nbr.data_ptr(), touch.data_ptr(), C.c_void_p(stream))
    if rc != abi.SFM_OK:
        raise SFMError(rc, "sfm_link_blocks")
    return parent, child, nbr, touch
