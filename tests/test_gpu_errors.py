"""Error paths of the C ABI on the GPU, made on the host side only.

- MOM_ERR_SINGULAR: a caller's matrix with a zero column (mom_gpu_set_matrix),
  the condition under which ZGETRF returns INFO > 0 and the reference STOPs
  (linalg.f90:170-173); also a column of NaN (no pivot candidate at all).
- MOM_ERR_NOCONV: mixed-precision refinement with one step and an
  unreachable tolerance.
- MOM_ERR_TIMEOUT: the bounded device waits given a limit of one poll
  (mom_gpu_set_wait_limits) for the LU panel exchange, the tensor-core GEMM's
  mbarriers and the triangular solve's hand-offs, one at a time.  A kernel
  that gives up records the error, waits for its own copies and tensor-core
  work, frees its tensor memory and returns; the test then checks that the
  same context, with the default limits, solves correctly again.
No test here faults or hangs the GPU: every failure is a bounded wait that a
limit ends, or a matrix the host builds.
"""
import os

import numpy as np
import pytest

import mom_b200 as M
from mom_b200 import workloads as W

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
WL = 600e-9
SRC = [M.src_pw(0, 90, 0)]


@pytest.fixture(scope="module")
def small(built):
    s = M.Solver(0)
    nodes, faces, ids, doms = W.sphere(1)
    s.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    yield s
    s.close()


@pytest.mark.parametrize("prec", [M.FP64, M.MIXED])
def test_singular_matrix(small, prec):
    om = M.omega_of(WL)
    ri = [1.0, np.sqrt(W.EPS_AU)]
    A = small.sysmat(om, ri, M.FP64, want_host=True)
    q = small.srcvec(om, ri[0], SRC, want_host=True)
    for bad in (0.0, np.nan):
        Ab = A.copy()
        Ab[:, 17] = bad
        small.set_matrix(Ab, prec)
        with pytest.raises(M.MomError) as e:
            small.solve(prec, tol=1e-12, maxit=30)
        assert e.value.status == M.MOM_ERR_SINGULAR
    # the same context factors the intact matrix afterwards
    small.set_matrix(A, prec)
    x = small.solve(prec, tol=1e-12, maxit=30)
    xr = np.linalg.solve(A, q)
    assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)


def test_refinement_no_convergence(small):
    om = M.omega_of(WL)
    ri = [1.0, np.sqrt(W.EPS_AU)]
    with pytest.raises(M.MomError) as e:
        small.solve_wavelength(om, ri, SRC, M.MIXED, 1e-300, 1)
    assert e.value.status == M.MOM_ERR_NOCONV
    small.solve_wavelength(om, ri, SRC, M.MIXED, 1e-12, 30)


def test_bounded_waits_time_out_and_recover(built):
    """cfg1 sphere (3840 unknowns) with the one-cluster panel kernel off
    (MOM_PANEL_CLUSTER=0, read when the context is created; with it, every
    mixed panel of this order fits one cluster, which has no spin-wait): the
    panels use the device-wide exchange, the trailing updates the tensor-core
    GEMM."""
    ref = np.load(os.path.join(HERE, "golden", "oracle_sphere_s3.npz"))
    os.environ["MOM_PANEL_CLUSTER"] = "0"
    try:
        s = M.Solver(0)
    finally:
        del os.environ["MOM_PANEL_CLUSTER"]
    try:
        nodes, faces, ids, doms = W.sphere(3)
        s.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
        om = M.omega_of(WL)
        ri = [1.0, np.sqrt(W.EPS_AU)]

        def ext():
            s.solve_wavelength(om, ri, SRC, M.MIXED, 1e-12, 30, want_host=False)
            a, b = s.cross_sections(om, ri[0], SRC)
            return a[0] + b[0]

        assert abs(ext() - ref["sigma"][2]) <= 1e-6 * ref["sigma"][2]  # autotune + graph capture
        for limits, what in (((1, 0, 0), "panel"), ((0, 1, 0), "tensor-core"), ((0, 0, 1), "triangular solve")):
            s.set_wait_limits(*limits)
            with pytest.raises(M.MomError) as e:
                ext()
            assert e.value.status == M.MOM_ERR_TIMEOUT, (limits, str(e.value))
            assert what in str(e.value), (limits, str(e.value))
            s.set_wait_limits(0, 0, 0)
            assert abs(ext() - ref["sigma"][2]) <= 1e-6 * ref["sigma"][2], limits
    finally:
        s.close()
