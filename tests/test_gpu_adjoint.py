"""Adjoint gradients against central finite differences of the GPU FP64 cross
sections (through the C ABI).

Steps follow the finite-difference protocol of the adjoint configuration:
1e-6 in eps (real and imaginary parts) and 1e-4 nm in vertex coordinates.
Tolerance: 1e-5 relative (eps), and 1e-5 of the gradient's largest entry
(vertices, where single entries can be near zero).
"""
import numpy as np
import pytest

import mom_b200 as M
from mom_b200 import meshgen

pytestmark = pytest.mark.gpu

WL = 600e-9
EPS = -9 + 1.3j
SRC = [M.src_pw(0, 90, 0)]


def sphere(s, perturbed):
    if perturbed:
        nodes, faces = meshgen.perturbed_sphere(s, 50.0, lmax=4, sigma=0.03, seed=4)
    else:
        nodes, faces = meshgen.icosphere(s, 50.0)
    return nodes, faces, np.ones(len(faces), int), [[1], [-1]]


def core_shell(s):
    n1, f1 = meshgen.icosphere(s, 40.0)
    n2, f2 = meshgen.icosphere(s, 60.0)
    nodes = np.vstack([n1, n2])
    faces = np.vstack([f1, f2 + len(n1)])
    ids = np.r_[np.full(len(f1), 1), np.full(len(f2), 2)]
    return nodes, faces, ids, [[2], [-2, 1], [-1]]


@pytest.fixture(scope="module")
def solver(built):
    s = M.Solver(0)
    yield s
    s.close()


def sigmas(S, geo, ri, prec=M.FP64, srcs=SRC):
    nodes, faces, ids, doms = geo
    S.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    om = M.omega_of(WL)
    S.solve_wavelength(om, ri, srcs, prec, 1e-12, 30)
    csca, cabs = S.cross_sections(om, ri[0], srcs)
    return np.stack([csca + cabs, cabs], axis=1)  # [nsrc][ext, abs]


def ri_of(eps_list):
    return [1.0] + [np.sqrt(e) for e in eps_list]


@pytest.mark.parametrize("prec", [M.FP64, M.MIXED])
def test_eps_gradient_matches_fd(solver, prec):
    geo = sphere(1, perturbed=True)
    ri = ri_of([EPS])
    sigmas(solver, geo, ri, prec)
    g = solver.adjoint(M.omega_of(WL), ri, SRC, prec, eps_dom=1)["deps"][0]  # [ext, abs][Re, Im]
    h = 1e-6
    for j, dz in enumerate([h, 1j * h]):
        sp = sigmas(solver, geo, ri_of([EPS + dz]))[0]
        sm = sigmas(solver, geo, ri_of([EPS - dz]))[0]
        fd = (sp - sm) / (2 * h)
        for k in range(2):
            assert abs(g[k, j] - fd[k]) <= 1e-5 * abs(fd[k]), (prec, j, k, g[k, j], fd[k])


def test_eps_gradient_plain_geometry_matches_dual(solver, monkeypatch):
    """The permittivity gradient of adj_eps_kernel (FP64 geometry, dual numbers
    in k only) equals that of the all-dual adj_pair_kernel (MOM_ADJ_EPS_PLAIN=0),
    on one and on several objectives and with the dense-W contraction."""
    geo = core_shell(1)
    ri = ri_of([EPS, 2.13])
    srcs = [M.src_pw(30, 40, 0), M.src_pw_elliptic(120, 250, 0.3 + 0.4j)]
    om = M.omega_of(WL)
    sigmas(solver, geo, ri, M.FP64, srcs)
    plain = solver.adjoint(om, ri, srcs, M.FP64, eps_dom=1)["deps"]
    plain_mean = solver.adjoint_mean_eps(om, ri, srcs, M.FP64, eps_dom=1)
    monkeypatch.setenv("MOM_ADJ_EPS_PLAIN", "0")
    other = M.Solver(0)
    try:
        sigmas(other, geo, ri, M.FP64, srcs)
        dual = other.adjoint(om, ri, srcs, M.FP64, eps_dom=1)["deps"]
        dual_mean = other.adjoint_mean_eps(om, ri, srcs, M.FP64, eps_dom=1)
    finally:
        other.close()
    assert np.allclose(plain, dual, rtol=1e-11, atol=0), np.max(np.abs(plain / dual - 1))
    assert np.allclose(plain_mean, dual_mean, rtol=1e-11, atol=0)


def test_vertex_gradient_plain_partners_matches_dual(solver, monkeypatch):
    """Vertex gradients of adj_vertex_kernel (the seeded face dual, partner faces
    in plain FP64) equal those of the all-dual adj_pair_kernel
    (MOM_ADJ_VERTEX_PLAIN=0) on the perturbed s=2 sphere, two objectives."""
    geo = sphere(2, perturbed=True)
    ri = ri_of([EPS])
    srcs = [M.src_pw(0, 90, 0), M.src_pw_elliptic(50, 20, 1j)]
    om = M.omega_of(WL)
    sigmas(solver, geo, ri, M.FP64, srcs)
    plain = solver.adjoint(om, ri, srcs, M.FP64, nodes=True)["dnodes"]
    monkeypatch.setenv("MOM_ADJ_VERTEX_PLAIN", "0")
    other = M.Solver(0)
    try:
        sigmas(other, geo, ri, M.FP64, srcs)
        dual = other.adjoint(om, ri, srcs, M.FP64, nodes=True)["dnodes"]
    finally:
        other.close()
    for a, b in zip(plain, dual):
        scale = np.abs(b).max()
        assert np.abs(a - b).max() <= 1e-11 * scale, np.abs(a - b).max() / scale


def test_eps_gradient_core_shell_mean(solver):
    """d(mean sigma)/d(shell eps) over several incidences, dense-W contraction."""
    geo = core_shell(1)
    eps_core = 2.13
    srcs = [M.src_pw(30, 40, 0), M.src_pw_elliptic(120, 250, 0.3 + 0.4j), M.src_pw(75, 300, 20)]
    ri = ri_of([EPS, eps_core])
    s0 = sigmas(solver, geo, ri, M.FP64, srcs)
    gm = solver.adjoint_mean_eps(M.omega_of(WL), ri, srcs, M.FP64, eps_dom=1)
    # per-source gradients of the same quantity must average to the mean
    per = []
    for s in srcs:
        sigmas(solver, geo, ri, M.FP64, [s])
        per.append(solver.adjoint(M.omega_of(WL), ri, [s], M.FP64, eps_dom=1)["deps"][0])
    assert np.allclose(np.mean(per, axis=0), gm, rtol=1e-9, atol=0)
    h = 1e-6
    for j, dz in enumerate([h, 1j * h]):
        sp = sigmas(solver, geo, ri_of([EPS + dz, eps_core]), M.FP64, srcs).mean(axis=0)
        sm = sigmas(solver, geo, ri_of([EPS - dz, eps_core]), M.FP64, srcs).mean(axis=0)
        fd = (sp - sm) / (2 * h)
        for k in range(2):
            assert abs(gm[k, j] - fd[k]) <= 1e-5 * abs(fd[k]), (j, k, gm[k, j], fd[k])
    assert s0.shape == (3, 2)


@pytest.mark.parametrize("prec", [M.FP64, M.MIXED])
def test_vertex_gradient_matches_fd(solver, prec):
    geo = sphere(1, perturbed=True)
    nodes, faces, ids, doms = geo
    ri = ri_of([EPS])
    sigmas(solver, geo, ri, prec)
    prob = M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms)
    out = solver.adjoint(M.omega_of(WL), ri, SRC, prec, nodes=True)
    # master-mesh gradient per nm: sum the domains' node entries
    gm = np.zeros((2, len(nodes), 3))
    for d, gd in enumerate(out["dnodes"]):
        par = prob.node_parent(d)
        np.add.at(gm, (slice(None), par), gd[0] * 1e-9)
    rng = np.random.default_rng(7)
    picks = [(int(v), int(k)) for v, k in zip(rng.choice(len(nodes), 6, replace=False), rng.integers(0, 3, 6))]
    h = 1e-4  # nm
    scale = np.abs(gm).max(axis=(1, 2))
    for v, k in picks:
        npl = nodes.copy()
        npl[v, k] += h
        nmi = nodes.copy()
        nmi[v, k] -= h
        sp = sigmas(solver, (npl, faces, ids, doms), ri)[0]
        sm = sigmas(solver, (nmi, faces, ids, doms), ri)[0]
        fd = (sp - sm) / (2 * h)
        for o in range(2):
            assert abs(gm[o, v, k] - fd[o]) <= 1e-5 * scale[o], (prec, v, k, o, gm[o, v, k], fd[o])


@pytest.mark.parametrize("prec", [M.FP64, M.MIXED])
def test_matches_oracle_finite_differences(solver, prec):
    """Against central differences of the oracle's own cross sections
    (tests/golden/adjoint_fd_s1.json, made by make_adjoint_fd.py)."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "adjoint_fd_s1.json")) as fh:
        ref = json.load(fh)
    geo = sphere(1, perturbed=True)
    nodes, faces, ids, doms = geo
    eps = complex(*ref["eps"])
    ri = ri_of([eps])
    s = sigmas(solver, geo, ri, prec)[0]
    assert np.allclose(s, ref["sigma"], rtol=1e-9 if prec == M.FP64 else 1e-6)
    out = solver.adjoint(M.omega_of(WL), ri, SRC, prec, eps_dom=1, nodes=True)
    g = out["deps"][0]
    for j in range(2):
        for k in range(2):
            fd = ref["deps"][j][k]
            assert abs(g[k, j] - fd) <= 1e-5 * abs(fd), (j, k, g[k, j], fd)
    prob = M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms)
    gm = np.zeros((2, len(nodes), 3))
    for d, gd in enumerate(out["dnodes"]):
        np.add.at(gm, (slice(None), prob.node_parent(d)), gd[0] * 1e-9)
    scale = np.abs(gm).max(axis=(1, 2))
    for v, k, fd in ref["dverts"]:
        for o in range(2):
            assert abs(gm[o, v, k] - fd[o]) <= 1e-5 * scale[o], (v, k, o, gm[o, v, k], fd[o])


def test_autograd_wrapper_gradcheck(solver):
    """torch.autograd.gradcheck of the autograd wrapper (mom_b200.autograd): its
    backward (one adjoint call) against torch's own central differences of the
    forward (FP64 solves) in eps and in every node coordinate of the s=1
    perturbed sphere; cross sections normalised by their value at the start."""
    import torch
    from mom_b200 import autograd as AG
    nodes, faces, ids, doms = sphere(1, perturbed=True)
    om = M.omega_of(WL)
    ri = ri_of([EPS])
    s0 = sigmas(solver, (nodes, faces, ids, doms), ri)[0]
    scale = torch.tensor(1.0 / s0, dtype=torch.float64)

    def f(er, ei, nd):
        return AG.cross_sections(solver, er, ei, nd, faces, ids, doms, 1, om, ri, SRC[0], M.FP64) * scale

    er = torch.tensor(EPS.real, dtype=torch.float64, requires_grad=True)
    ei = torch.tensor(EPS.imag, dtype=torch.float64, requires_grad=True)
    nd = torch.tensor(nodes, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(f, (er, ei, nd), eps=1e-6, atol=1e-8, rtol=1e-5)
