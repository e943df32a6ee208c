"""Golden fixtures (tests/golden/, written by tests/golden/make_golden.py).

CPU: the oracle reproduces every fixture bit for bit (digest of the whole
interior potential, the sampled potential and g_x, the outer iteration
count and the ratio history).  GPU: the FP64 CUDA path reproduces the
periodic fixtures bit for bit and the isolated-sphere fixture to 1e-13
relative (its multipole moments are summed per block on the device, in a
different order).
"""
import os

import numpy as np
import pytest

from code_only_b200 import abi
from code_only_b200.solver import FMGPoisson
from tests.golden.make_golden import CASES, case_inputs, digest, interiors
from tests.oracle_lib import oracle_solve

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _fixture(name):
    with np.load(os.path.join(HERE, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_reproduces_fixture(name):
    fx = _fixture(name)
    h, p, rho = case_inputs(name)
    rc, psi, g, st, _ = oracle_solve(h, rho, p)
    assert rc == abi.SFM_OK
    phi = interiors(h, psi, p.ngh_io)
    assert digest(phi) == str(fx["sha256"])
    assert np.array_equal(phi.ravel()[fx["index"]], fx["psi"])
    assert np.array_equal(interiors(h, g[:, 0], p.ngh_io).ravel()[fx["index"]], fx["gx"])
    assert st.outer_iters == int(fx["outer_iters"])
    assert np.array_equal(np.array(st.history()), fx["ratio"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_gpu_fp64_reproduces_fixture(name):
    fx = _fixture(name)
    h, p, rho = case_inputs(name)
    with FMGPoisson(h, params=p) as s:
        psi, g, st = s.solve(rho)
    phi = interiors(h, psi, p.ngh_io).ravel()[fx["index"]]
    gx = interiors(h, g[:, 0], p.ngh_io).ravel()[fx["index"]]
    assert st.outer_iters == int(fx["outer_iters"])
    if p.bc == abi.SFM_BC_PERIODIC:
        assert digest(interiors(h, psi, p.ngh_io)) == str(fx["sha256"])
        assert np.array_equal(phi, fx["psi"]) and np.array_equal(gx, fx["gx"])
    else:
        assert np.abs(phi - fx["psi"]).max() <= 1e-13 * np.abs(fx["psi"]).max()
        assert np.abs(gx - fx["gx"]).max() <= 1e-13 * np.abs(fx["gx"]).max()
