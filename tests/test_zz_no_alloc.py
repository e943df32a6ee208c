"""sfm_uniform_solve_noalloc, the uniform periodic base-grid solve that
allocates nothing, against the full solve of the same problem through the
existing entry point (sfm_solve on a one-level periodic hierarchy).

Both converge the same 7-point periodic problem lap(phi) = 4 pi (rho - mean)
on the same grid, so after removing the free constant they agree to the
convergence tolerance: 1e-8 relative (max norm) with both solves run to a
relative residual of 1e-12.  Two calls in a row must both pass, and give
identical results (the kernel clears its fixed scratch itself).  The file
name puts it after every other GPU test; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

from code_only_b200 import abi, workloads as w
from code_only_b200.solver import FMGPoisson

pytestmark = pytest.mark.gpu

TOL = 1e-8
REL_TOL = 1e-12


def _entry(lib):
    f = lib.sfm_uniform_solve_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                  C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_void_p]
    f.restype = C.c_int
    return f


def _dense(h, a, g):
    """block array [nb, G, G, G] (x fastest) of a one-level hierarchy ->
    dense [n, n, n] indexed [k, j, i]"""
    ni = h.ni
    n = h.ngb[0] * ni
    out = np.empty((n, n, n))
    for b in range(h.nblocks):
        i, j, k = (int(v) * ni for v in h.ijk[b])
        out[k:k + ni, j:j + ni, i:i + ni] = a[b, g:g + ni, g:g + ni, g:g + ni]
    return out


def _rel_centered(a, b):
    a = a - a.mean()
    b = b - b.mean()
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("nbase,ni", [(2, 8), (4, 8)])
def test_noalloc_matches_full_solve_twice(nbase, ni):
    import torch
    h = w.uniform_periodic(nbase, ni)
    p = abi.default_params(abi.SFM_BC_PERIODIC, rel_tol=REL_TOL, max_outer=60)
    rho = w.block_field(h, p.ngh_io, w.gaussian_peak)
    with FMGPoisson(h, params=p) as s:
        psi_blocks, _, st = s.solve(rho, want_g=False)
    assert st.true_rel_residual <= 10 * REL_TOL
    ref = _dense(h, psi_blocks, p.ngh_io)
    n = ref.shape[0]
    hcell = float(h.cellwidth[0])

    f = _entry(abi.load_library())
    dev = torch.device("cuda:0")
    rho_d = torch.from_numpy(np.ascontiguousarray(_dense(h, rho, p.ngh_io))).to(dev)
    stream = torch.cuda.current_stream(dev)
    results = []
    for _ in range(2):
        psi_d = torch.full_like(rho_d, float("nan"))   # every entry must be written
        cycles, rr = C.c_int(-1), C.c_double(-1.0)
        rc = f(rho_d.data_ptr(), psi_d.data_ptr(), n, hcell, p.four_pi_G, REL_TOL, 200,
               C.byref(cycles), C.byref(rr), C.c_void_p(stream.cuda_stream))
        assert rc == abi.SFM_OK, abi.load_library().sfm_strerror(rc)
        assert 0 < cycles.value <= 200 and 0.0 <= rr.value <= REL_TOL
        out = psi_d.cpu().numpy()
        assert np.isfinite(out).all()
        assert _rel_centered(out, ref) <= TOL
        results.append(out)
    assert np.array_equal(results[0], results[1])


def test_noalloc_queues_without_host_outputs():
    import torch
    f = _entry(abi.load_library())
    n = 16
    rng = np.random.default_rng(7)
    rho = torch.from_numpy(rng.standard_normal((n, n, n))).cuda()
    psi_a = torch.empty_like(rho)
    psi_b = torch.empty_like(rho)
    stream = torch.cuda.current_stream()
    assert f(rho.data_ptr(), psi_a.data_ptr(), n, 1.0 / n, 1.0, 1e-10, 100, None, None,
             C.c_void_p(stream.cuda_stream)) == abi.SFM_OK
    cycles, rr = C.c_int(), C.c_double()
    assert f(rho.data_ptr(), psi_b.data_ptr(), n, 1.0 / n, 1.0, 1e-10, 100, C.byref(cycles), C.byref(rr),
             C.c_void_p(stream.cuda_stream)) == abi.SFM_OK
    assert torch.equal(psi_a, psi_b)


def test_noalloc_rejects_bad_arguments():
    import torch
    f = _entry(abi.load_library())
    a = torch.zeros(64 ** 3, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    args = (1.0 / 32, 1.0, 1e-10, 10, None, None, None)
    assert f(a.data_ptr(), b.data_ptr(), 64, *args) == abi.SFM_ESIZE      # above the fixed maximum
    assert f(a.data_ptr(), b.data_ptr(), 12, *args) == abi.SFM_ESIZE      # not a power of two
    assert f(a.data_ptr(), b.data_ptr(), 1, *args) == abi.SFM_ESIZE
    assert f(None, b.data_ptr(), 32, *args) == abi.SFM_EINVAL
    host = np.zeros(32 ** 3)
    assert f(host.ctypes.data, b.data_ptr(), 32, *args) == abi.SFM_EINVAL  # not device memory
    assert f(a.data_ptr() + 4, b.data_ptr(), 32, *args) == abi.SFM_EINVAL  # misaligned
    assert f(a.data_ptr(), b.data_ptr(), 32, -1.0, 1.0, 1e-10, 10, None, None, None) == abi.SFM_EINVAL


def test_noalloc_nonfinite_density_is_reported():
    """A NaN in rho must not come back as a converged zero potential: psi is
    all NaN and the call returns SFM_ENONFINITE with a cycle count of -1."""
    import torch
    f = _entry(abi.load_library())
    n = 16
    rho = torch.ones((n, n, n), dtype=torch.float64, device="cuda")
    rho[3, 5, 7] = float("nan")
    psi = torch.zeros_like(rho)
    cycles, rr = C.c_int(0), C.c_double(0.0)
    rc = f(rho.data_ptr(), psi.data_ptr(), n, 1.0 / n, 1.0, 1e-10, 100, C.byref(cycles), C.byref(rr),
           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == abi.SFM_ENONFINITE
    assert cycles.value == -1 and np.isnan(rr.value)
    assert torch.isnan(psi).all()
    # the next call on clean data is unaffected
    rho[3, 5, 7] = 2.0
    rc = f(rho.data_ptr(), psi.data_ptr(), n, 1.0 / n, 1.0, 1e-10, 100, C.byref(cycles), C.byref(rr),
           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == abi.SFM_OK and torch.isfinite(psi).all()


def test_noalloc_refuses_host_outputs_under_capture():
    """Host outputs need a wait, which stream capture forbids: the call
    returns SFM_EINVAL and leaves the capture intact."""
    import torch
    f = _entry(abi.load_library())
    n = 8
    rho = torch.ones((n, n, n), dtype=torch.float64, device="cuda")
    psi = torch.zeros_like(rho)
    s = torch.cuda.Stream()
    # a first call outside capture looks up the scratch array
    assert f(rho.data_ptr(), psi.data_ptr(), n, 1.0 / n, 1.0, 1e-10, 10, None, None,
             C.c_void_p(s.cuda_stream)) == abi.SFM_OK
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    cycles = C.c_int(0)
    with torch.cuda.graph(g, stream=s, capture_error_mode="thread_local"):
        rc = f(rho.data_ptr(), psi.data_ptr(), n, 1.0 / n, 1.0, 1e-10, 10, C.byref(cycles), None,
               C.c_void_p(s.cuda_stream))
        psi.add_(1.0)   # the capture is still usable after the refusal
    assert rc == abi.SFM_EINVAL and cycles.value == 0
