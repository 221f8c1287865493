"""The oracle's restatement of the second-harmonic branch (oracle.shg_solve:
nlsurf_coef nlsurf.f90:137-338, rwg_moments rwgf.f90:148-221,
determine_epsp solver.f90:393-433, sysmat_pmchwt_nls sysmat.f90:112-229)
against properties that do not depend on the reference being run:

- the RWG Gram matrix equals its closed form (the polar moment of each face
  about its centroid), which the 13-point rule integrates exactly up to its
  single-precision weights (they sum to 1 - 7.5e-9): 1e-7 relative;
- the second-harmonic far field of a sphere vanishes along the propagation
  axis, forwards and backwards (the selection rule of second-harmonic
  scattering from centrosymmetric spheres), for each susceptibility alone;
- nlx is linear in the susceptibilities and quadratic in the fundamental
  field;
- with no incident field the extinction vanishes (sigma_sca = -sigma_abs);
- determine_epsp takes the permittivity of the other domain of each face
  (a face in no other domain cannot occur: the decomposition check of
  submesh_edge_connectivity, mesh.f90:415-418, rejects such problems)."""
import numpy as np
import pytest

import oracle as O
from mom_b200 import workloads as W

WL = 1000e-9
SHRI = [1.0, np.sqrt(complex(-2.0, 3.5))]
RI = [1.0, np.sqrt(W.EPS_AU)]
SRC = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)


@pytest.fixture(scope="module")
def sphere1():
    nodes, faces, ids, doms = W.sphere(1)
    P = O.OracleProblem(nodes, faces, ids, 1e-9, doms)
    om = O.omega_of(WL)
    x = O.solve(P.sysmat(om, RI), P.srcvec(om, 1.0, SRC)[:, None])
    return P, om, x


def gram_closed_form(g):
    """<f_m, f_n> from the polar moment J = A (a^2 + b^2 + c^2) / 36 of each face
    about its centroid c: the integral of (r - v_q) . (r - v_p) is
    J + A (c - v_q) . (c - v_p)."""
    m = g["m"]
    nodes, fn = m["nodes"], m["face_node"]
    Nd = len(m["edge_node"])
    F = np.zeros((Nd, Nd))
    for f in range(g["F"]):
        p = nodes[fn[f]]
        c = p.mean(axis=0)
        A = g["A"][f]
        J = A * sum(np.sum((p[i] - p[(i + 1) % 3]) ** 2) for i in range(3)) / 36.0
        for q in range(3):
            for r in range(3):
                kq = g["sign"][f, q] * g["len"][f, q] / (2 * A)
                kr = g["sign"][f, r] * g["len"][f, r] / (2 * A)
                F[g["edge"][f, q], g["edge"][f, r]] += kq * kr * (J + A * np.dot(c - g["free"][f, q],
                                                                                 c - g["free"][f, r]))
    return F


@pytest.mark.parametrize("d", [0, 1])
def test_gram_matrix_closed_form(sphere1, d):
    P, _, _ = sphere1
    g = O._domain_geometry(P, d, O.tri_rule())
    Fm = O.rwg_moments(g)
    Fc = gram_closed_form(g)
    assert np.abs(Fm - Fc).max() <= 1e-7 * np.abs(Fc).max()
    assert np.array_equal(Fm, Fm.T)
    assert np.linalg.eigvalsh(Fm).min() > 0
    assert max(np.count_nonzero(row) for row in Fm) <= 5


@pytest.mark.parametrize("k", range(3))
def test_shg_axial_null(sphere1, k):
    P, om, x = sphere1
    chi = [0.0, 0.0, 0.0]
    chi[k] = 1e-18
    nlx = O.shg_solve(P, om, RI, SHRI, [None, tuple(chi)], x)
    r = P.rcs(2 * om, 1.0, nlx[:, 0], 19, 4)
    assert r.max() > 0
    assert r[0].max() <= 1e-10 * r.max() and r[-1].max() <= 1e-10 * r.max()


def test_shg_scaling(sphere1):
    P, om, x = sphere1
    chi = (1e-18 + 0.2e-18j, 0.4e-18, -0.3e-18j)
    a = O.shg_solve(P, om, RI, SHRI, [None, chi], x)
    b = O.shg_solve(P, om, RI, SHRI, [None, tuple(3 * c for c in chi)], x)
    c = O.shg_solve(P, om, RI, SHRI, [None, chi], 2 * x)
    assert np.linalg.norm(b - 3 * a) <= 1e-12 * np.linalg.norm(a)
    assert np.linalg.norm(c - 4 * a) <= 1e-12 * np.linalg.norm(a)
    csca, cabs = P.cs(2 * om, SHRI[0], a[:, 0], dict(type="none"))
    assert csca != 0 and abs(csca + cabs) <= 1e-12 * abs(csca)


def test_epsp(sphere1):
    P, _, _ = sphere1
    e = O.epsp_of(P, 1, RI)
    assert np.allclose(e, O.EPS0 * complex(RI[0]) ** 2, rtol=0, atol=0)
    e = O.epsp_of(P, 0, RI)
    assert np.allclose(e, O.EPS0 * complex(RI[1]) ** 2, rtol=1e-15, atol=0)


def test_shg_with_mirror_group_reproduces_full_sphere():
    """The second harmonic of the eighth of the mirror-symmetric s=1 sphere with
    the group mxp x myp x mzp (the boundary conditions of edge_bc on the plane
    edges, the polarisation projected on each representation) equals the full
    sphere's without a group: SH cross sections through cs_prtsrf with no
    incident field."""
    from mom_b200 import meshgen
    nodes, faces = meshgen.octasphere(1, 50.0)
    om = O.omega_of(WL)
    chi = (1e-18 + 0.3e-18j, 0.5e-18, -0.2e-18)
    src = dict(type="pw", theta=0.4, phi=0.3, psi=0.2)
    full = O.OracleProblem(nodes, faces, np.ones(len(faces), int), 1e-9, [[1], [-1]])
    x = O.solve(full.sysmat(om, RI), full.srcvec(om, 1.0, src)[:, None])
    nlx = O.shg_solve(full, om, RI, SHRI, [None, chi], x)
    ref = full.cs(2 * om, SHRI[0], nlx[:, 0], dict(type="none"))
    fn, ff, lines = meshgen.symmetry_fragment(nodes, faces, [0, 1, 2])
    Q = O.OracleProblem(fn, ff, np.ones(len(ff), int), 1e-9, [[1], [-1]])
    Q.set_symmetry(["mxp", "myp", "mzp"])
    for ax, name in enumerate(("xplane", "yplane", "zplane")):
        Q.classify_edges(lines[ax], name)
    A = Q.sysmat_sym(om, RI)
    xs = Q.solve_sym(A, Q.srcvec_sym(om, 1.0, src))
    Q_nlx = O.shg_solve_sym(Q, om, RI, SHRI, [None, chi], xs)
    got = Q.cs_sym(2 * om, SHRI[0], Q_nlx, dict(type="none"))
    assert abs(got[0] / ref[0] - 1) <= 1e-10 and abs(got[1] / ref[1] - 1) <= 1e-10, (got, ref)
