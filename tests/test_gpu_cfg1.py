"""Full-size parity at the plain-FP64 single-solve configuration (icosphere
s=3, 3840 unknowns): the GPU FP64 path against the oracle's committed outputs
(tests/golden/oracle_sphere_s3.npz, made by tests/golden/make_cfg1.py).
Tolerances: PMCHWT block Frobenius norms and the whole-matrix product A v
<= 1e-10 relative, RHS <= 1e-12, solution, cross sections and far field
<= 1e-9; mixed precision sigma_ext <= 1e-6."""
import os

import numpy as np
import pytest

import mom_b200 as M
from mom_b200 import workloads as W

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def ref():
    return np.load(os.path.join(HERE, "golden", "oracle_sphere_s3.npz"))


@pytest.fixture(scope="module")
def solver(built):
    s = M.Solver(0)
    nodes, faces, ids, doms = W.sphere(3)
    s.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    yield s
    s.close()


def test_fp64_full_size_parity(solver, ref):
    om = M.omega_of(600e-9)
    ri = [1.0, np.sqrt(W.EPS_AU)]
    src = [M.src_pw(0, 90, 0)]
    A = solver.sysmat(om, ri, M.FP64, want_host=True)
    N = A.shape[0] // 2
    blocks = [np.linalg.norm(A[:N, :N]), np.linalg.norm(A[N:, N:]), np.linalg.norm(A[N:, :N]),
              np.linalg.norm(A[:N, N:])]
    assert np.all(np.abs(np.array(blocks) - ref["blocks"]) <= 1e-10 * ref["blocks"])
    rng = np.random.default_rng(1234)
    v = rng.standard_normal(2 * N) + 1j * rng.standard_normal(2 * N)
    assert rel(A @ v, ref["Av"]) <= 1e-10
    q = solver.srcvec(om, ri[0], src, want_host=True)
    assert rel(q[:, 0], ref["q"]) <= 1e-12
    x = solver.solve(M.FP64, want_host=True)
    assert rel(x[:, 0], ref["x"]) <= 1e-9
    csca, cabs = solver.cross_sections(om, ri[0], src)
    sig = np.array([csca[0], cabs[0], csca[0] + cabs[0]])
    assert np.all(np.abs(sig - ref["sigma"]) <= 1e-9 * np.abs(ref["sigma"]))
    rcs = solver.rcs(om, ri[0], 91, 180)
    assert rel(rcs[::5, ::9], ref["rcs_sub"]) <= 1e-9
    assert abs(np.linalg.norm(rcs) - ref["rcs_norm"]) <= 1e-9 * ref["rcs_norm"]


def test_mixed_full_size_sigma(solver, ref):
    om = M.omega_of(600e-9)
    ri = [1.0, np.sqrt(W.EPS_AU)]
    src = [M.src_pw(0, 90, 0)]
    solver.solve_wavelength(om, ri, src, M.MIXED, 1e-12, 30)
    csca, cabs = solver.cross_sections(om, ri[0], src)
    assert abs(csca[0] + cabs[0] - ref["sigma"][2]) <= 1e-6 * ref["sigma"][2]
