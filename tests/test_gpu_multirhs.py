"""Many right-hand sides (the GEMM-based blocked solve, used from 16 columns
on; with the mixed path's FP32 factors from 64 columns on the 256-row blocked
solve with tensor-core updates) against the single-column cooperative solve,
for A x = b and, through the adjoint, A^T x = b; FP64 and mixed (both refined
to 1e-12)."""
import numpy as np
import pytest

import mom_b200 as M
from mom_b200 import workloads as W

pytestmark = pytest.mark.gpu

WL = 600e-9


@pytest.fixture(scope="module")
def solver(built):
    s = M.Solver(0)
    nodes, faces, ids, doms = W.core_shell(1)
    s.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    yield s
    s.close()


RI = [1.0, np.sqrt(W.EPS_AU), np.sqrt(W.EPS_SILICA)]


@pytest.mark.parametrize("ns", [20, 70])
@pytest.mark.parametrize("prec", [M.FP64, M.MIXED])
def test_multi_rhs_solve_matches_single(solver, prec, ns):
    srcs = W.incidences(ns)
    om = M.omega_of(WL)
    X = solver.solve_wavelength(om, RI, srcs, prec, 1e-12, 30, want_host=True)
    for k in (0, 7, ns - 1):
        x1 = solver.solve_wavelength(om, RI, [srcs[k]], prec, 1e-12, 30, want_host=True)[:, 0]
        err = np.linalg.norm(X[:, k] - x1) / np.linalg.norm(x1)
        assert err <= (1e-12 if prec == M.FP64 else 1e-10), (prec, k, err)


@pytest.mark.parametrize("ns", [10, 35])  # 20 or 70 transposed right-hand sides
@pytest.mark.parametrize("prec", [M.FP64, M.MIXED])
def test_multi_rhs_transposed_solve_through_adjoint(solver, prec, ns):
    srcs = W.incidences(ns)
    om = M.omega_of(WL)
    solver.solve_wavelength(om, RI, srcs, prec, 1e-12, 30)
    gm = solver.adjoint_mean_eps(om, RI, srcs, prec, eps_dom=1)
    per = []
    for s in srcs[:3]:
        solver.solve_wavelength(om, RI, [s], prec, 1e-12, 30)
        per.append(solver.adjoint(om, RI, [s], prec, eps_dom=1)["deps"][0])
    solver.solve_wavelength(om, RI, srcs[3:], prec, 1e-12, 30)
    rest = solver.adjoint_mean_eps(om, RI, srcs[3:], prec, eps_dom=1)
    mean = (np.sum(per, axis=0) + (ns - 3) * rest) / ns
    assert np.allclose(mean, gm, rtol=1e-8, atol=0), (mean, gm)
