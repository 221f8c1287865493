"""Full-size parity at the mixed-precision-at-scale configuration (icosphere
s=4, 5120 triangles, 15,360 unknowns, eps = -9 + 1.3i, 600 nm, x-polarised
plane wave along +z) against the oracle's FP64 outputs
(tests/golden/oracle_sphere_s4.npz, made by tests/golden/make_cfg2.py).

Tolerances: FP64 path -- PMCHWT block Frobenius norms and the whole-matrix
product A v <= 1e-10 relative, RHS <= 1e-12, solution and cross sections
<= 1e-9; mixed path -- sigma_ext, sigma_sca and sigma_abs <= 1e-6 relative
against the FP64 oracle (the headline accuracy bound)."""
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
    return np.load(os.path.join(HERE, "golden", "oracle_sphere_s4.npz"))


@pytest.fixture(scope="module")
def solver(built):
    s = M.Solver(0)
    nodes, faces, ids, doms = W.sphere(4)
    s.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    yield s
    s.close()


def test_fp64_cfg2_parity(solver, ref):
    om = M.omega_of(600e-9)
    ri = [1.0, np.sqrt(W.EPS_AU)]
    src = [M.src_pw(0, 90, 0)]
    A = solver.sysmat(om, ri, M.FP64, want_host=True)
    N = A.shape[0] // 2
    blocks = np.array([np.linalg.norm(A[:N, :N]), np.linalg.norm(A[N:, N:]), np.linalg.norm(A[N:, :N]),
                       np.linalg.norm(A[:N, N:])])
    assert np.all(np.abs(blocks - ref["blocks"]) <= 1e-10 * ref["blocks"]), blocks / ref["blocks"] - 1
    rng = np.random.default_rng(4321)
    v = rng.standard_normal(2 * N) + 1j * rng.standard_normal(2 * N)
    assert rel(A @ v, ref["Av"]) <= 1e-10
    del A
    q = solver.srcvec(om, ri[0], src, want_host=True)
    assert rel(q[:, 0], ref["q"]) <= 1e-12
    x = solver.solve(M.FP64, want_host=True)
    assert rel(x[:, 0], ref["x"]) <= 1e-9
    csca, cabs = solver.cross_sections(om, ri[0], src)
    sig = np.array([csca[0], cabs[0], csca[0] + cabs[0]])
    assert np.all(np.abs(sig - ref["sigma"]) <= 1e-9 * np.abs(ref["sigma"])), sig / ref["sigma"] - 1


def test_mixed_cfg2_sigma_against_fp64_oracle(solver, ref):
    om = M.omega_of(600e-9)
    ri = [1.0, np.sqrt(W.EPS_AU)]
    src = [M.src_pw(0, 90, 0)]
    solver.solve_wavelength(om, ri, src, M.MIXED, 1e-12, 60, want_host=False)
    csca, cabs = solver.cross_sections(om, ri[0], src)
    sig = np.array([csca[0], cabs[0], csca[0] + cabs[0]])
    assert np.all(np.abs(sig - ref["sigma"]) <= 1e-6 * np.abs(ref["sigma"])), sig / ref["sigma"] - 1
