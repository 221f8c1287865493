"""CPU checks of the oracle (the FP64 C restatement of the reference).

The reference ships no golden vectors and cannot be compiled here (no
Fortran compiler), so these tests pin the oracle by mathematics and physics:
closed-form singular integrals (int.f90) against dense numerical quadrature,
the triangle rules (quad.f90), the Mie series on the sphere, the lossless
limit sigma_abs -> 0, and a committed regression fixture of the oracle's own
output (tests/golden/oracle_sphere_s1.json, made by tests/golden/make_golden.py).
"""
import json
import os

import numpy as np
import pytest

import oracle as O
import mie
from mom_b200 import meshgen

HERE = os.path.dirname(os.path.abspath(__file__))


def sphere(s, r=50.0):
    nodes, faces = meshgen.icosphere(s, r)
    return nodes, faces, np.ones(len(faces), int)


@pytest.fixture(scope="module")
def p1():
    nodes, faces, ids = sphere(1)
    return O.OracleProblem(nodes, faces, ids, 1e-9, [[1], [-1]])


def test_constants_single_precision_pi():
    # constants.f90:10: pi is a default-real literal, rounded to single precision
    assert O.lib().oracle_pi() == float(np.float32(3.141592653589))
    assert O.PI_F != np.pi and abs(O.PI_F - np.pi) < 1e-7


@pytest.mark.parametrize("name,nq", [("tri_gl1", 1), ("tri_gl3", 3), ("tri_gl4", 4), ("tri_gl7", 7), ("tri_gl13", 13)])
def test_triangle_rules(name, nq):
    w, nd = O.tri_rule(name)
    assert len(w) == nq
    assert abs(w.sum() - 1.0) < 2e-7
    assert np.allclose(nd.sum(1), 1.0, atol=3e-7)


def test_gl13_is_single_precision_and_degree_7():
    w, nd = O.tri_rule("tri_gl13")
    # quad.f90:115-171 literals carry no _dp suffix
    assert np.all(w == w.astype(np.float32).astype(np.float64))
    assert np.all(nd == nd.astype(np.float32).astype(np.float64))
    # exact (to the float rounding of the literals) for x^a y^b, a + b <= 7, on the unit triangle
    from math import factorial
    x, y = nd[:, 0], nd[:, 1]
    for a in range(8):
        for b in range(8 - a):
            exact = factorial(a) * factorial(b) / factorial(a + b + 2) * 2  # divided by area 1/2
            assert abs((w * x ** a * y ** b).sum() - exact) < 5e-7


def _dense_rule(V, level=6):
    w13, n13 = O.tri_rule("tri_gl13")
    tris = [tuple(V)]
    for _ in range(level):
        new = []
        for a, b, c in tris:
            ab, bc, ca = (a + b) / 2, (b + c) / 2, (c + a) / 2
            new += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        tris = new
    pts, wts = [], []
    for a, b, c in tris:
        ar = 0.5 * np.linalg.norm(np.cross(b - a, c - a))
        for t in range(13):
            pts.append(n13[t, 2] * a + n13[t, 0] * b + n13[t, 1] * c)
            wts.append(w13[t] * ar)
    return np.array(pts), np.array(wts)


@pytest.mark.parametrize("where", ["offplane", "inplane_outside"])
def test_closed_form_singular_integrals(p1, where):
    """int.f90 (Hanninen 2006 forms) against dense quadrature at non-singular points:
    K2m1 = int f/R, K21 = int f R, K1m1 = int div f / R, K11 = int div f R,
    K4m1 = int (r-r')/R^3 x f, K41 = -int (r-r')/R x f."""
    f_idx = 5
    g = p1.face_geometry(0, f_idx)
    V, area = g["nodes"], g["area"]
    cen = V.mean(0)
    nrm = np.cross(V[1] - V[0], V[2] - V[0])
    nrm /= np.linalg.norm(nrm)
    L = np.linalg.norm(V[1] - V[0])
    if where == "offplane":
        r = cen + 0.3 * L * nrm + 0.2 * L * (V[0] - cen) / np.linalg.norm(V[0] - cen)
    else:
        r = V[0] + 0.5 * (V[0] - cen)
    pts, wts = _dense_rule(V)
    for e in range(3):
        res = p1.static_integrals(0, r, f_idx, e)
        sgn, le, p = g["sign"][e], g["length"][e], g["bnode"][e]
        f = sgn * le / (2 * area) * (pts - p)
        d = r - pts
        R = np.linalg.norm(d, axis=1)
        num = dict(K2m1=(wts[:, None] * f / R[:, None]).sum(0), K21=(wts[:, None] * f * R[:, None]).sum(0),
                   K1m1=(wts * sgn * le / area / R).sum(), K11=(wts * sgn * le / area * R).sum(),
                   K4m1=(wts[:, None] * np.cross(d / R[:, None] ** 3, f)).sum(0),
                   K41=-(wts[:, None] * np.cross(d / R[:, None], f)).sum(0))
        for k, v in num.items():
            err = np.linalg.norm(np.atleast_1d(res[k] - v))
            # (r - p) x K3 can vanish by symmetry; assess K4m1 / K41 on the scale of the f/R, f R terms
            scale = {"K4m1": np.linalg.norm(num["K2m1"]) / L, "K41": np.linalg.norm(num["K21"]) / L}.get(k, 0.0)
            assert err <= 1e-6 * max(np.linalg.norm(np.atleast_1d(v)), scale), (k, e, err)


def test_mie_convergence():
    """sigma_ext of the faceted sphere approaches the Mie series as the mesh is refined."""
    wl = 600e-9
    n2 = np.sqrt(-9 + 1.3j)
    ext_mie = mie.mie_cross_sections(50e-9, wl, n2)[0]
    errs = []
    for s in (1, 2):
        nodes, faces, ids = sphere(s)
        P = O.OracleProblem(nodes, faces, ids, 1e-9, [[1], [-1]])
        om = O.omega_of(wl)
        src = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)
        x = O.solve(P.sysmat(om, [1.0, n2]), P.srcvec(om, 1.0, src))
        sca, ab = P.cs(om, 1.0, x, src)
        errs.append(abs(sca + ab - ext_mie) / ext_mie)
    assert errs[1] < errs[0] and errs[1] < 0.08, errs


def test_lossless_absorption_vanishes_under_refinement():
    errs = []
    for s in (1, 2):
        nodes, faces, ids = sphere(s)
        P = O.OracleProblem(nodes, faces, ids, 1e-9, [[1], [-1]])
        om = O.omega_of(600e-9)
        src = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)
        x = O.solve(P.sysmat(om, [1.0, 1.5]), P.srcvec(om, 1.0, src))
        sca, ab = P.cs(om, 1.0, x, src)
        errs.append(abs(ab / sca))
    assert errs[1] < 0.6 * errs[0] and errs[1] < 0.01, errs


def test_oracle_regression_fixture(p1):
    with open(os.path.join(HERE, "golden", "oracle_sphere_s1.json")) as fh:
        g = json.load(fh)
    om = O.omega_of(g["wavelength"])
    ri = [complex(*v) for v in g["ri"]]
    A = p1.sysmat(om, ri)
    assert abs(np.linalg.norm(A) - g["A_frobenius"]) <= 1e-12 * g["A_frobenius"]
    for (i, j, re, im) in g["A_entries"]:
        assert abs(A[i, j] - complex(re, im)) <= 1e-12 * abs(complex(re, im)) + 1e-30
    src = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)
    x = O.solve(A, p1.srcvec(om, ri[0], src))
    sca, ab = p1.cs(om, ri[0], x, src)
    assert abs(sca - g["csca"]) <= 1e-10 * abs(g["csca"])
    assert abs(ab - g["cabs"]) <= 1e-10 * abs(g["cabs"])


def test_adjoint_fd_fixture_is_the_oracles():
    """tests/golden/adjoint_fd_s1.json holds central differences of this oracle's
    cross sections: recompute sigma and the d/dRe(eps) entry."""
    with open(os.path.join(HERE, "golden", "adjoint_fd_s1.json")) as fh:
        g = json.load(fh)
    nodes, faces = meshgen.perturbed_sphere(1, 50.0, lmax=4, sigma=0.03, seed=4)
    ids = np.ones(len(faces), int)
    src = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)
    om = O.omega_of(g["wavelength"])
    eps = complex(*g["eps"])

    def sig(e):
        P = O.OracleProblem(nodes, faces, ids, 1e-9, [[1], [-1]])
        ri = [1.0 + 0j, complex(np.sqrt(e))]
        x = O.solve(P.sysmat(om, ri), P.srcvec(om, ri[0], src))
        sca, ab = P.cs(om, ri[0], x, src)
        return np.array([sca + ab, ab])

    assert np.allclose(sig(eps), g["sigma"], rtol=1e-10)
    h = g["deps_step"]
    fd = (sig(eps + h) - sig(eps - h)) / (2 * h)
    assert np.allclose(fd, g["deps"][0], rtol=1e-8)


# ---- near fields (nfields.f90 scat_fields), pinned by physics ----

@pytest.fixture(scope="module")
def s2_solution():
    """The s=2 gold sphere (960 unknowns) solved by the oracle at 600 nm."""
    from mom_b200 import workloads as W
    nodes, faces, ids, doms = W.sphere(2)
    P = O.OracleProblem(nodes, faces, ids, 1e-9, doms)
    om = O.omega_of(600e-9)
    n_in = np.sqrt(W.EPS_AU)
    src = dict(type="pw", theta=0.0, phi=90 * O.PI_F / 180, psi=0.0)
    A = P.sysmat(om, np.array([1.0, n_in]))
    x = O.solve(A, P.srcvec(om, 1.0, src)[:, None])[:, 0]
    return P, om, n_in, src, x, np.asarray(nodes) * 1e-9, np.asarray(faces)


def test_near_field_matches_far_field_at_one_metre(s2_solution):
    """At r = 1 m the scattered |E|^2 equals the rcs routine's value (ffields.f90)
    in the same direction, to O(size / r)."""
    P, om, n_in, src, x, _, _ = s2_solution
    rcs = P.rcs(om, 1.0, x, 19, 37)
    for th, it in ((0.0, 0), (float(O.PI_F), 18)):
        e, _ = P.scat_fields(om, 1.0, x, [[np.sin(th), 0.0, np.cos(th)]], d=0)
        assert abs(np.sum(np.abs(e[0, 0]) ** 2) / rcs[it, 0] - 1) < 1e-6


def test_extinction_theorem_and_null_field(s2_solution):
    """Inside the particle the exterior representation cancels the incident field,
    and outside it the interior representation vanishes (to the s=2 discretisation)."""
    P, om, n_in, src, x, _, _ = s2_solution
    inside = [[0, 0, 0], [10e-9, 5e-9, -8e-9]]
    e, _ = P.scat_fields(om, 1.0, x, inside, srcs=[src], d=0)
    einc, _ = P.scat_fields(om, 1.0, np.zeros_like(x), inside, srcs=[src], d=0)
    assert np.abs(e).max() < 2e-2 * np.abs(einc).max()
    outside = [[0, 0, 120e-9], [80e-9, 0, 0]]
    e2, _ = P.scat_fields(om, n_in, x, outside, d=1)
    es, _ = P.scat_fields(om, 1.0, x, outside, d=0)
    assert np.abs(e2).max() < 5e-3 * np.abs(es).max()


def test_normal_field_jump_at_the_surface(s2_solution):
    """Just outside / inside a face centroid (0.01 edge lengths along the face
    normal, the singular integrals in use) eps_out E_n^out = eps_in E_n^in and the
    tangential H is continuous, to a few per cent."""
    P, om, n_in, src, x, nodes, faces = s2_solution
    eps_in = n_in ** 2
    for fi in (0, 17, 100):
        tri = nodes[faces[fi]]
        cp = tri.mean(axis=0)
        nn = np.cross(tri[1] - tri[0], tri[2] - tri[0])
        nn /= np.linalg.norm(nn)
        nn = nn if np.dot(nn, cp) > 0 else -nn
        d = 0.01 * np.linalg.norm(tri[1] - tri[0])
        eo, ho = P.scat_fields(om, 1.0, x, [cp + d * nn], srcs=[src], d=0)
        ei, hi = P.scat_fields(om, n_in, x, [cp - d * nn], d=1)
        ratio = np.dot(eo[0, 0], nn) / (eps_in * np.dot(ei[0, 0], nn))
        assert abs(ratio - 1) < 0.05
        tan = lambda v: v - np.dot(v, nn) * nn
        assert np.linalg.norm(tan(ho[0, 0]) - tan(hi[0, 0])) < 0.06 * np.linalg.norm(tan(ho[0, 0]))


# ---- symmetry groups (read_symm, sbnd, bc.f90), mirror planes ----

def _octa(s):
    nodes, faces = meshgen.octasphere(s, 50.0)
    return nodes, faces


@pytest.mark.parametrize("s,tol", [(1, 1e-12), (2, 1e-8)])
def test_symmetry_fragments_reproduce_the_full_sphere(s, tol):
    """The half, quarter and eighth of a mirror-symmetric sphere, solved per
    representation with the mirror groups and the symmetry-plane boundary
    conditions, give the cross sections of the full sphere (the same
    discretisation; at s=2 the near-pair threshold, 3 average edge lengths of the
    fragment's own mesh, differs slightly from the full mesh's)."""
    nodes, faces = _octa(s)
    om = O.omega_of(600e-9)
    n_in = np.sqrt(complex(-9, 1.3))
    srcs = [dict(type="pw", theta=0.3, phi=0.7, psi=0.4), dict(type="pw_elliptic", theta=1.1, phi=-0.4, phase=1j)]
    P = O.OracleProblem(nodes, faces, np.ones(len(faces), int), 1e-9, [[1], [-1]])
    A = P.sysmat(om, np.array([1.0, n_in]))
    ref = []
    for src in srcs:
        x = O.solve(A, P.srcvec(om, 1.0, src)[:, None])[:, 0]
        ref.append(P.cs(om, 1.0, x, src))
    for planes, names in (([0], ["mxp"]), ([0, 1], ["mxp", "myp"]), ([0, 1, 2], ["mxp", "myp", "mzp"])):
        fn, ff, lines = meshgen.symmetry_fragment(nodes, faces, planes)
        Q = O.OracleProblem(fn, ff, np.ones(len(ff), int), 1e-9, [[1], [-1]])
        assert Q.set_symmetry(names) == 2 ** len(planes)
        for ax in planes:
            assert Q.classify_edges(lines[ax], ["xplane", "yplane", "zplane"][ax]) == len(lines[ax])
        As = Q.sysmat_sym(om, [1.0, n_in])
        for src, (csca, cabs) in zip(srcs, ref):
            xs = Q.solve_sym(As, Q.srcvec_sym(om, 1.0, src))
            a, b = Q.cs_sym(om, 1.0, xs, src)
            assert abs(a / csca - 1) < tol and abs(b / cabs - 1) < tol


def test_mirror_group_structure_and_boundary_conditions():
    """symmetry.f90 product_group: orthogonal characters, det J = +-1; bc.f90
    edge_bc removes, per representation, J on the plane edges where the mirror's
    field action is +1 and M where its action times det J is +1."""
    nodes, faces = _octa(1)
    fn, ff, lines = meshgen.symmetry_fragment(nodes, faces, [0, 1])
    Q = O.OracleProblem(fn, ff, np.ones(len(ff), int), 1e-9, [[1], [-1]])
    n = Q.set_symmetry(["mxp", "myp"])
    j, detj, ef = Q.group_info()
    assert n == 4 and np.allclose(np.abs(detj), 1)
    assert np.allclose(ef.conj().T @ ef, n * np.eye(n))
    for a in range(n):
        assert np.allclose(j[a] @ j[a].T, np.eye(3)) and np.isclose(np.linalg.det(j[a]), detj[a])
    Q.classify_edges(lines[0], "xplane")
    Q.classify_edges(lines[1], "yplane")
    N = Q.N
    for r in range(n):
        idv, _ = Q.edge_bc(r)
        # a plane edge loses exactly one of J, M in each representation
        assert np.count_nonzero(idv == -1) == len(lines[0]) + len(lines[1])
        assert np.all(idv[:N][idv[N:] == -1] == 0)


def test_field_mesh_matches_near_fields_at_the_surface():
    """field_mesh (nfpost.f90:167-262) gives the fields on the surface from the
    currents alone; they must agree with the integrated fields (scat_fields, plus
    the incident field outside) a hundredth of an edge off the surface, on either
    side, to the discretisation error of the s=2 sphere (measured 1-8%)."""
    from mom_b200 import workloads as W
    nodes, faces, ids, doms = W.sphere(2)
    P = O.OracleProblem(nodes, faces, ids, 1e-9, doms)
    om = O.omega_of(600e-9)
    n_in = np.sqrt(W.EPS_AU)
    src = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)
    x = O.solve(P.sysmat(om, np.array([1.0, n_in])), P.srcvec(om, 1.0, src)[:, None])
    e, h = O.field_mesh(P, 0, om, 1.0, x[:, 0])
    ei, hi = O.field_mesh(P, 1, om, n_in, x[:, 0])
    nd = np.asarray(nodes) * 1e-9
    fc = np.asarray(faces)
    for f in (7, 100, 250):
        tri = nd[fc[f]]
        cp = tri.mean(axis=0)
        nn = np.cross(tri[1] - tri[0], tri[2] - tri[0])
        nn = nn / np.linalg.norm(nn) * np.sign(nn @ cp)
        dh = 0.01 * np.linalg.norm(tri[1] - tri[0])
        eo, ho = P.scat_fields(om, 1.0, x, np.array([cp + dh * nn]), srcs=[src], d=0)
        en, hn = P.scat_fields(om, n_in, x, np.array([cp - dh * nn]), d=1)
        for a, b, tol in ((e[f], eo[0, 0], 0.12), (h[f], ho[0, 0], 0.05), (ei[f], en[0, 0], 0.05),
                          (hi[f], hn[0, 0], 0.02)):
            assert np.linalg.norm(a - b) <= tol * np.linalg.norm(b), (f, np.linalg.norm(a - b) / np.linalg.norm(b))
