"""Near fields on the GPU (mom_gpu_scat_fields, nfields.f90 scat_fields) against
the oracle: the same currents (the oracle's FP64 solution of the s=2 gold
sphere), points far away, just outside and inside the surface (singular
integrals in use) and in the interior domain, with and without the incident
field.  FP64 on both sides: relative difference <= 1e-9."""
import numpy as np
import pytest

import mom_b200 as M
import oracle as O
from mom_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(built):
    nodes, faces, ids, doms = W.sphere(2)
    P = O.OracleProblem(nodes, faces, ids, 1e-9, doms)
    om = M.omega_of(600e-9)
    n_in = np.sqrt(W.EPS_AU)
    srcs = [M.src_pw(0, 90, 0), M.src_pw_elliptic(35, 20, np.exp(0.4j))]
    A = P.sysmat(om, np.array([1.0, n_in]))
    q = np.stack([P.srcvec(om, 1.0, s) for s in srcs], axis=1)
    x = O.solve(A, q)
    S = M.Solver(0)
    S.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    nd = np.asarray(nodes) * 1e-9
    fc = np.asarray(faces)
    tri = nd[fc[7]]
    cp = tri.mean(axis=0)
    nn = np.cross(tri[1] - tri[0], tri[2] - tri[0])
    nn = nn / np.linalg.norm(nn) * np.sign(np.dot(nn, cp))
    h = np.linalg.norm(tri[1] - tri[0])
    outside = np.array([[0, 0, 1.0], [0.3, -0.2, 0.5], [0, 0, 80e-9], cp + 0.02 * h * nn, cp + 0.5 * h * nn])
    inside = np.array([[0, 0, 0], [10e-9, -5e-9, 20e-9], cp - 0.02 * h * nn])
    yield P, S, om, n_in, srcs, x, outside, inside
    S.close()


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("with_incident", [False, True])
def test_exterior_fields_match_oracle(setup, with_incident):
    P, S, om, n_in, srcs, x, outside, _ = setup
    sr = srcs if with_incident else None
    e, h = S.scat_fields(om, 1.0, outside, x=x, srcs=sr, dom=0)
    eo, ho = P.scat_fields(om, 1.0, x, outside, srcs=sr, d=0)
    for k in range(len(outside)):  # per point: the far points are 1e7 times weaker
        assert rel(e[:, k], eo[:, k]) <= 1e-9
        assert rel(h[:, k], ho[:, k]) <= 1e-9


def test_interior_fields_match_oracle(setup):
    P, S, om, n_in, srcs, x, _, inside = setup
    e, h = S.scat_fields(om, n_in, inside, x=x, dom=1)
    eo, ho = P.scat_fields(om, n_in, x, inside, d=1)
    for k in range(len(inside)):
        assert rel(e[:, k], eo[:, k]) <= 1e-9
        assert rel(h[:, k], ho[:, k]) <= 1e-9


def test_device_solutions_give_the_same_fields(setup):
    """After a GPU solve, the device solutions (x=None) and the same solutions
    copied to the host give identical fields."""
    P, S, om, n_in, srcs, x, outside, _ = setup
    xg = S.solve_wavelength(om, [1.0, n_in], srcs, M.FP64, 1e-12, 30)
    e1, h1 = S.scat_fields(om, 1.0, outside, nsrc=2, dom=0)
    e2, h2 = S.scat_fields(om, 1.0, outside, x=xg, dom=0)
    assert np.array_equal(e1, e2) and np.array_equal(h1, h2)
    assert rel(xg, x) <= 1e-9  # and they agree with the oracle's solution
