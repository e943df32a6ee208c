"""Writes the golden fixtures of tests/golden/ from the oracle.

The reference ships no golden vectors for the FMG solve, so these fixtures
pin the CPU restatement (oracle/) on small seeded inputs: any later change
to the oracle's arithmetic or pass order shows up as a fixture mismatch, and
the GPU FP64 path is compared against the same numbers.  Each case stores the
SHA-256 of the potential on block interiors (float64, C order: a bitwise
pin), 2048 seeded samples of the potential and of g_x with their flat
indices (for tolerance checks and diagnosis), the outer iteration count and
the ratio history, at the reference's default tolerances (errormax 1e-3, nfmgmax 10)
and, for the isolated sphere, the reference's l <= 3 multipoles.

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from code_only_b200 import abi, workloads as w  # noqa: E402
from tests.oracle_lib import oracle_solve  # noqa: E402

CASES = {
    "uniform16_periodic": (lambda: w.uniform_periodic(2, 8), w.gaussian_peak, abi.SFM_BC_PERIODIC, {}),
    "amr2_periodic": (lambda: w.small_periodic(2, 8, 2, 0), w.gaussian_peak, abi.SFM_BC_PERIODIC, {}),
    "amr2_sphere_l3": (lambda: w.small_sphere(2, 8, 2, 0), w.softened_sphere, abi.SFM_BC_SPHERE, {"zero_mean": 0}),
}


def case_inputs(name):
    mk, fn, bc, kw = CASES[name]
    h = mk()
    p = abi.default_params(bc, **kw)
    rho = w.block_field(h, p.ngh_io, fn)
    return h, p, rho


def interiors(h, a, g):
    n = h.ni
    return np.ascontiguousarray(a[:, g:g + n, g:g + n, g:g + n])


NSAMPLE = 2048


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def sample_index(size):
    return np.sort(np.random.default_rng(2024).choice(size, NSAMPLE, replace=False))


def main():
    for name in CASES:
        h, p, rho = case_inputs(name)
        rc, psi, g, st, _ = oracle_solve(h, rho, p)
        assert rc == abi.SFM_OK, (name, rc)
        phi = interiors(h, psi, p.ngh_io)
        gx = interiors(h, g[:, 0], p.ngh_io)
        idx = sample_index(phi.size)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"),
                            sha256=np.array(digest(phi)), index=idx,
                            psi=phi.ravel()[idx], gx=gx.ravel()[idx],
                            outer_iters=np.int32(st.outer_iters),
                            ratio=np.array(st.history(), dtype=np.float64))
        print(name, "iters", st.outer_iters, "ratios", st.history())


if __name__ == "__main__":
    main()
