"""ctypes loader of the CPU restatement in oracle/ (the checker)."""
import ctypes as C
import os
import subprocess

import numpy as np

from code_only_b200 import abi, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")

_lib = None
# the exchange callback of oracle_solve_split: (user, kind, f, L, dir, data, n)
XCHG_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_int64)


def load_oracle():
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(ORACLE_DIR, "sfmg_oracle.cpp")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    lib = C.CDLL(ORACLE_SO)
    lib.oracle_solve.argtypes = [C.POINTER(abi.SfmHierDesc), C.POINTER(abi.SfmParams), C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.POINTER(abi.SfmStats), C.c_int, C.c_void_p]
    lib.oracle_solve.restype = C.c_int
    lib.oracle_check_linklist.argtypes = [C.POINTER(abi.SfmHierDesc)]
    lib.oracle_check_linklist.restype = C.c_int
    lib.oracle_apply_L.argtypes = [C.POINTER(abi.SfmHierDesc), C.POINTER(abi.SfmParams), C.c_void_p, C.c_void_p]
    lib.oracle_apply_L.restype = C.c_int
    lib.oracle_threads.restype = C.c_int
    lib.oracle_multipole.argtypes = [C.POINTER(abi.SfmHierDesc), C.POINTER(abi.SfmParams), C.c_void_p, C.c_int,
                                     C.c_void_p, C.c_void_p]
    lib.oracle_multipole.restype = C.c_int
    lib.oracle_apply_LT.argtypes = [C.POINTER(abi.SfmHierDesc), C.POINTER(abi.SfmParams), C.c_void_p, C.c_void_p]
    lib.oracle_apply_LT.restype = C.c_int
    lib.oracle_adjoint.argtypes = [C.POINTER(abi.SfmHierDesc), C.POINTER(abi.SfmParams), C.c_void_p, C.c_void_p,
                                   C.POINTER(abi.SfmStats)]
    lib.oracle_adjoint.restype = C.c_int
    lib.oracle_ghost_pass.argtypes = [C.POINTER(abi.SfmHierDesc), C.POINTER(abi.SfmParams), C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_void_p]
    lib.oracle_ghost_pass.restype = C.c_int
    lib.oracle_step.argtypes = [C.POINTER(abi.SfmHierDesc), C.POINTER(abi.SfmParams), C.c_int, C.c_int, C.c_int,
                                C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p]
    lib.oracle_step.restype = C.c_int
    lib.oracle_relax.argtypes = [C.POINTER(abi.SfmHierDesc), C.POINTER(abi.SfmParams), C.c_int, C.c_int,
                                 C.c_void_p, C.c_void_p, C.c_void_p]
    lib.oracle_relax.restype = C.c_int
    lib.oracle_solve_split.argtypes = [C.POINTER(abi.SfmHierDesc), C.POINTER(abi.SfmParams), C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.POINTER(abi.SfmStats), C.c_void_p, XCHG_FN, C.c_void_p]
    lib.oracle_solve_split.restype = C.c_int
    lib.oracle_profile.argtypes = [C.POINTER(abi.SfmHierDesc), C.POINTER(abi.SfmParams), C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.POINTER(abi.SfmStats), C.c_void_p]
    lib.oracle_profile.restype = C.c_int
    _lib = lib
    return lib


def oracle_solve(h, rho, params, psi=None, want_g=True, stage=0):
    """Runs the oracle; returns (rc, psi, g, stats, dump)."""
    lib = load_oracle()
    d = abi.HierDesc(h)
    psi = np.zeros_like(rho) if psi is None else np.array(psi, dtype=np.float64, copy=True)
    g = np.zeros((h.nblocks, 3) + rho.shape[1:]) if want_g else None
    st = abi.SfmStats()
    G1 = h.ni + 2
    dump = np.zeros((h.nblocks, G1, G1, G1)) if stage else None
    rc = lib.oracle_solve(d.ref(), C.byref(params), np.ascontiguousarray(rho).ctypes.data, psi.ctypes.data,
                          g.ctypes.data if g is not None else None, C.byref(st), stage,
                          dump.ctypes.data if dump is not None else None)
    return rc, psi, g, st, dump


def oracle_adjoint(h, dJ_dphi, params):
    """Runs the oracle's adjoint; returns (rc, dJ_drho, stats)."""
    lib = load_oracle()
    out = np.zeros_like(dJ_dphi)
    st = abi.SfmStats()
    rc = lib.oracle_adjoint(abi.HierDesc(h).ref(), C.byref(params), np.ascontiguousarray(dJ_dphi).ctypes.data,
                            out.ctypes.data, C.byref(st))
    return rc, out, st


def leaf_mask(h, n_ghost):
    """bool [nb, G, G, G]: interior cells of leaf blocks (blocks whose fields the solve determines)"""
    G = h.ni + 2 * n_ghost
    m = np.zeros((h.nblocks, G, G, G), bool)
    leaf = (h.level == h.nlev - 1) | (h.child[:, 0] < 0)
    m[leaf, n_ghost:n_ghost + h.ni, n_ghost:n_ghost + h.ni, n_ghost:n_ghost + h.ni] = True
    return m


def make_rho(h, fn, ngh):
    return workloads.block_field(h, ngh, fn)


def oracle_ghost_pass(h, field, f, L=-1, d=0, cubic=False):
    """One ghost pass (AMR level L, direction d) at fmg level f on `field`
    ([nb, G, G, G], G = (ni >> f) + 2) in place, or the whole fill when L < 0."""
    lib = load_oracle()
    assert field.dtype == np.float64 and field.flags.c_contiguous
    rc = lib.oracle_ghost_pass(abi.HierDesc(h).ref(), C.byref(abi.default_params(abi.SFM_BC_PERIODIC)), f, L, d,
                               1 if cubic else 0, field.ctypes.data)
    assert rc == 0, rc


# pieces of the composite operator (oracle_step)
(STEP_CONVERGE, STEP_BOUNDARY_U, STEP_GHOST, STEP_FLUX, STEP_FLUXCORR, STEP_RESID, STEP_RELAX, STEP_BASE_SOLVE,
 STEP_P2C) = range(9)


def _ptr(a):
    if a is None:
        return None
    assert a.flags.c_contiguous
    return a.ctypes.data


def oracle_step(h, step, f, u=None, flux=None, rhs=None, out=None, L=0, d=0, flag=0, own=None,
                bc=abi.SFM_BC_PERIODIC):
    """One piece of the composite operator at fmg level f, for the blocks with
    own[b] (all blocks when own is None); arrays [nb, G, G, G] updated in
    place, flux a list of the three face-flux arrays."""
    lib = load_oracle()
    G = (h.ni >> f) + 2
    for a in [u, rhs, None if step == STEP_RELAX else out] + list(flux or []):   # relax: out[0] = max
        assert a is None or (a.dtype == np.float64 and a.size == h.nblocks * G ** 3), "array of the wrong size"
    own8 = None if own is None else np.ascontiguousarray(own, dtype=np.int8)
    fx, fy, fz = flux if flux is not None else (None, None, None)
    rc = lib.oracle_step(abi.HierDesc(h).ref(), C.byref(abi.default_params(bc)), step, f, L, d,
                         flag, _ptr(own8), _ptr(u), _ptr(fx), _ptr(fy), _ptr(fz), _ptr(rhs), _ptr(out))
    assert rc == 0, rc


def oracle_relax(h, u, rhs, f, sweeps):
    """`sweeps` red-black sweeps of fmg_poisson_relax on u in place; returns Resh2maxg."""
    lib = load_oracle()
    G = (h.ni >> f) + 2
    assert u.size == rhs.size == h.nblocks * G ** 3, "array of the wrong size"
    m = C.c_double(0.0)
    rc = lib.oracle_relax(abi.HierDesc(h).ref(), C.byref(abi.default_params(abi.SFM_BC_PERIODIC)), f, sweeps,
                          _ptr(u), _ptr(np.ascontiguousarray(rhs)), C.byref(m))
    assert rc == 0, rc
    return m.value


def oracle_solve_split(h, rho, params, owner, rank, exchanges):
    """The oracle's solve on this rank's blocks (owner == rank), the other
    ranks' values filled in through `exchanges(kind, f, L, d, array)` before
    every step that reads them (see Oracle::xchg).  Returns (rc, psi, g,
    stats); psi and g hold the owned blocks' results."""
    lib = load_oracle()
    own = np.ascontiguousarray(owner == rank, dtype=np.int8)
    psi = np.zeros_like(rho)
    g = np.zeros((h.nblocks, 3) + rho.shape[1:])
    st = abi.SfmStats()
    errors = []

    def cb(user, kind, f, L, d, data, n):
        try:
            exchanges(kind, f, L, d, np.ctypeslib.as_array(data, shape=(n,)))
        except Exception as e:   # an exception cannot cross the C frames: record it
            errors.append(e)
            raise

    fn = XCHG_FN(cb)
    rc = lib.oracle_solve_split(abi.HierDesc(h).ref(), C.byref(params), np.ascontiguousarray(rho).ctypes.data,
                                psi.ctypes.data, g.ctypes.data, C.byref(st), own.ctypes.data, fn, None)
    if errors:
        raise errors[0]
    return rc, psi, g, st


PROFILE_CLASSES = ("other", "ghost passes", "converge", "face fluxes", "flux correction", "relaxation",
                   "residuals", "restriction", "prolongation", "base grid", "physical boundary", "psi2g")


def oracle_profile(h, rho, params):
    """One oracle solve with the exclusive wall time of each routine class;
    returns (rc, {class: seconds}, total seconds, stats)."""
    lib = load_oracle()
    psi = np.zeros_like(rho)
    g = np.zeros((h.nblocks, 3) + rho.shape[1:])
    secs = np.zeros(len(PROFILE_CLASSES) + 1)
    st = abi.SfmStats()
    rc = lib.oracle_profile(abi.HierDesc(h).ref(), C.byref(params), np.ascontiguousarray(rho).ctypes.data,
                            psi.ctypes.data, g.ctypes.data, C.byref(st), secs.ctypes.data)
    return rc, dict(zip(PROFILE_CLASSES, secs[:-1].tolist())), float(secs[-1]), st
