"""Symmetry groups of mirror planes on the GPU (read_symm, sbnd, edge_bc and the
nga > 1 branches of sysmat_pmchwt, srcvec, solve_systems, cs_prtsrf and
far_fields), through the C ABI, against the oracle's restatement.

The half, quarter and eighth of a mirror-symmetric sphere (the octahedron
sphere, whose coordinate planes are mirror planes of the mesh), with the
plane edges classified by sbnd and the groups mxp, mxp x myp, mxp x myp x mzp:
- every representation's matrix (the unknowns the boundary conditions keep)
  matches the oracle's sysmat with the group to 1e-10 (relative Frobenius);
- right-hand sides to 1e-12, solutions to 1e-9, cross sections to 1e-9;
- the cross sections equal those of the full sphere solved without symmetry
  (the same discretisation; at s=3 to 1e-8, the oracle's own agreement level,
  because the near-pair threshold follows each fragment's mean edge length);
- mixed precision: cross sections to 1e-6;
- the far field of the fragment with its group equals the full sphere's.
"""
import numpy as np
import pytest

import mom_b200 as M
import oracle as O
from mom_b200 import meshgen

pytestmark = pytest.mark.gpu

WL = 600e-9
N_IN = np.sqrt(complex(-9, 1.3))
SRCS = [dict(type="pw", theta=0.3, phi=0.7, psi=0.4), dict(type="pw_elliptic", theta=1.1, phi=-0.4, phase=1j)]
CASES = [([0], ["mxp"]), ([0, 1], ["mxp", "myp"]), ([0, 1, 2], ["mxp", "myp", "mzp"])]
PLANES = ["xplane", "yplane", "zplane"]


def gpu_src(d):
    if d["type"] == "pw":
        return M.src_pw(d["theta"] / M.DEGTORAD, d["phi"] / M.DEGTORAD, d["psi"] / M.DEGTORAD)
    return M.src_pw_elliptic(d["theta"] / M.DEGTORAD, d["phi"] / M.DEGTORAD, d["phase"])


def fragment(s, planes):
    nodes, faces = meshgen.octasphere(s, 50.0)
    fn, ff, lines = meshgen.symmetry_fragment(nodes, faces, planes)
    return fn, ff, lines


def gpu_problem(fn, ff, lines, planes):
    prob = M.Problem.from_arrays(fn, ff, np.ones(len(ff), int), 1e-9, [[1], [-1]])
    ln = np.concatenate([np.asarray(lines[ax], dtype=np.int32).reshape(-1, 2) for ax in planes])
    ids = np.concatenate([np.full(len(lines[ax]), 10 + ax, np.int32) for ax in planes])
    prob.set_lines(ln, ids)
    for ax in planes:
        assert prob.classify_edges(10 + ax, PLANES[ax]) == len(lines[ax])
    return prob


def oracle_problem(fn, ff, lines, planes, names):
    Q = O.OracleProblem(fn, ff, np.ones(len(ff), int), 1e-9, [[1], [-1]])
    Q.set_symmetry(names)
    for ax in planes:
        Q.classify_edges(lines[ax], PLANES[ax])
    return Q


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def solver(built):
    s = M.Solver(0)
    yield s
    s.close()


@pytest.mark.parametrize("case", range(3))
def test_fragment_matches_oracle(solver, case):
    planes, names = CASES[case]
    fn, ff, lines = fragment(2, planes)
    prob = gpu_problem(fn, ff, lines, planes)
    solver.set_problem(prob)
    nga = solver.set_symmetry(names, prob)
    assert nga == 2 ** len(planes)
    Q = oracle_problem(fn, ff, lines, planes, names)
    om = M.omega_of(WL)
    ri = [1.0, N_IN]
    A = solver.sysmat(om, ri, M.FP64, want_host=True)
    Ao = Q.sysmat_sym(om, [1.0, N_IN])
    for r in range(nga):
        idv, _ = Q.edge_bc(r)
        keep = np.nonzero(idv != -1)[0]
        sub = np.ix_(keep, keep)
        assert rel(A[r][sub], Ao[r][sub]) <= 1e-10, r
        rm = np.nonzero(idv == -1)[0]
        assert np.allclose(A[r][rm][:, rm], np.eye(len(rm)))  # identity rows for the removed unknowns
    for src in SRCS:
        q = solver.srcvec(om, ri[0], [gpu_src(src)], want_host=True)[:, :, 0]  # (2N, nga)
        qo = Q.srcvec_sym(om, 1.0, src)  # (nga, 2N)
        for r in range(nga):
            idv, _ = Q.edge_bc(r)
            keep = idv != -1
            assert rel(q[keep, r], qo[r][keep]) <= 1e-12, r
            assert np.all(q[~keep, r] == 0)
        x = solver.solve(M.FP64, want_host=True)[:, :, 0]
        xo = Q.solve_sym(Ao, qo)
        for r in range(nga):
            assert rel(x[:, r], xo[r]) <= 1e-9, r
        csca, cabs = solver.cross_sections(om, ri[0], [gpu_src(src)])
        so, ao = Q.cs_sym(om, 1.0, xo, src)
        assert abs(csca[0] - so) <= 1e-9 * abs(so) and abs(cabs[0] - ao) <= 1e-9 * abs(ao)
        # the same through host solutions
        c2, a2 = solver.cross_sections(om, ri[0], [gpu_src(src)], x=x[:, :, None])
        assert abs(c2[0] - csca[0]) <= 1e-13 * abs(csca[0]) and abs(a2[0] - cabs[0]) <= 1e-13 * abs(cabs[0])


@pytest.mark.parametrize("s,tol", [(1, 1e-11), (3, 1e-8)])
def test_fragments_reproduce_the_full_sphere(solver, s, tol):
    nodes, faces = meshgen.octasphere(s, 50.0)
    om = M.omega_of(WL)
    ri = [1.0, N_IN]
    srcs = [gpu_src(d) for d in SRCS]
    solver.set_problem(M.Problem.from_arrays(nodes, faces, np.ones(len(faces), int), 1e-9, [[1], [-1]]))
    solver.solve_wavelength(om, ri, srcs, M.FP64, want_host=False)
    ref = solver.cross_sections(om, ri[0], srcs)
    ff_ref = solver.rcs(om, ri[0], 19, 37, isrc=0)
    for planes, names in CASES:
        fn, ff, lines = fragment(s, planes)
        prob = gpu_problem(fn, ff, lines, planes)
        solver.set_problem(prob)
        solver.set_symmetry(names, prob)
        for prec, t in ((M.FP64, tol), (M.MIXED, max(tol, 1e-6))):
            solver.solve_wavelength(om, ri, srcs, prec, 1e-12, 30, want_host=False)
            csca, cabs = solver.cross_sections(om, ri[0], srcs)
            assert np.all(np.abs(csca / ref[0] - 1) < t) and np.all(np.abs(cabs / ref[1] - 1) < t), (names, prec)
            ffr = solver.rcs(om, ri[0], 19, 37, isrc=0)
            assert rel(ffr, ff_ref) < 10 * t, (names, prec)


def test_command_script_with_mirror_groups(solver, tmp_path):
    """The `mom` interpreter with symm 3 mxp myp mzp and sbnd on an eighth of the
    s=1 sphere (plane edges as Gmsh line elements): its .crs file matches the
    full sphere's cross sections to the printed EN15.3 precision."""
    import os
    import subprocess
    nodes, faces = meshgen.octasphere(1, 50.0)
    fn, ff, lines = fragment(1, [0, 1, 2])
    with open(tmp_path / "eighth.msh", "w") as fh:
        fh.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(fn))
        for i, p in enumerate(fn):
            fh.write("%d %.17g %.17g %.17g\n" % (i + 1, p[0], p[1], p[2]))
        ne = sum(len(lines[ax]) for ax in range(3)) + len(ff)
        fh.write("$EndNodes\n$Elements\n%d\n" % ne)
        k = 1
        for ax in range(3):
            for a, b in lines[ax]:
                fh.write("%d 1 2 %d %d %d %d\n" % (k, 10 + ax, 10 + ax, a + 1, b + 1))
                k += 1
        for f in ff:
            fh.write("%d 2 2 1 1 %d %d %d\n" % (k, f[0] + 1, f[1] + 1, f[2] + 1))
            k += 1
        fh.write("$EndElements\n")
    script = "\n".join([
        "name 'eighth'", "symm 3 mxp myp mzp", "mesh 'eighth.msh' 1d-9",
        "sbnd 10 xplane", "sbnd 11 yplane", "sbnd 12 zplane", "wlls 1 600d-9", "nmed 2",
        "smed 1 linear value (1.0, 0.0)", "smed 2 linear value (%.17g, %.17g)" % (N_IN.real, N_IN.imag),
        "ndom 2", "sdom 1 1 1 0 1 -1", "sdom 2 1 -1 0 2 -1", "fdom", "nsrc 1", "ssrc 1 'pw' 0 90 0",
        "solv", "crst", "exit"]) + "\n"
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "for90-mom2_b200", "bin",
                       "mom_b200")
    r = subprocess.run([exe], input=script, capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:]
    assert "Created a symmetry group with 8 elements." in r.stdout
    row = [float(v) for v in open(tmp_path / "eighth-s1.crs").read().split()]
    om = M.omega_of(WL)
    solver.set_problem(M.Problem.from_arrays(nodes, faces, np.ones(len(faces), int), 1e-9, [[1], [-1]]))
    src = [M.src_pw(0, 90, 0)]
    solver.solve_wavelength(om, [1.0, N_IN], src, M.FP64, want_host=False)
    csca, cabs = solver.cross_sections(om, 1.0, src)
    assert abs(row[1] - csca[0]) <= 5e-4 * csca[0] and abs(row[2] - cabs[0]) <= 5e-4 * cabs[0], (row, csca, cabs)


def test_command_script_second_harmonic_with_mirror_groups(solver, tmp_path):
    """The `mom` interpreter with symm 3 mxp myp mzp, sbnd and a surface
    nonlinearity (`smed 2 nlsurf value ...`) on the eighth of the s=1 sphere:
    its -sh.crs file matches the full sphere's second-harmonic cross sections
    (C ABI, no group) to the printed EN15.3 precision."""
    import os
    import subprocess
    chi = (1e-18 + 0.2e-18j, 0.5e-18, -0.3e-18)
    cx = lambda z: "(%.17g, %.17g)" % (complex(z).real, complex(z).imag)
    nodes, faces = meshgen.octasphere(1, 50.0)
    fn, ff, lines = fragment(1, [0, 1, 2])
    with open(tmp_path / "eighth.msh", "w") as fh:
        fh.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(fn))
        for i, p in enumerate(fn):
            fh.write("%d %.17g %.17g %.17g\n" % (i + 1, p[0], p[1], p[2]))
        ne = sum(len(lines[ax]) for ax in range(3)) + len(ff)
        fh.write("$EndNodes\n$Elements\n%d\n" % ne)
        k = 1
        for ax in range(3):
            for a, b in lines[ax]:
                fh.write("%d 1 2 %d %d %d %d\n" % (k, 10 + ax, 10 + ax, a + 1, b + 1))
                k += 1
        for f in ff:
            fh.write("%d 2 2 1 1 %d %d %d\n" % (k, f[0] + 1, f[1] + 1, f[2] + 1))
            k += 1
        fh.write("$EndElements\n")
    script = "\n".join([
        "name 'eighth'", "symm 3 mxp myp mzp", "mesh 'eighth.msh' 1d-9",
        "sbnd 10 xplane", "sbnd 11 yplane", "sbnd 12 zplane", "wlls 1 600d-9", "nmed 2",
        "smed 1 linear value (1.0, 0.0)", "smed 2 linear value " + cx(N_IN),
        "smed 2 nlsurf value " + " ".join(cx(c) for c in chi),
        "ndom 2", "sdom 1 1 1 0 1 -1", "sdom 2 1 -1 0 2 -1", "fdom", "nsrc 1", "ssrc 1 'pw' 0 90 0",
        "solv", "crst", "exit"]) + "\n"
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "for90-mom2_b200", "bin",
                       "mom_b200")
    r = subprocess.run([exe], input=script, capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:]
    assert "Solving nonlinear scattering from centrosymmetric material" in r.stdout
    row = [float(v) for v in open(tmp_path / "eighth-s1-sh.crs").read().split()]
    om = M.omega_of(WL)
    ri = [1.0, N_IN]
    src = [M.src_pw(0, 90, 0)]
    solver.set_problem(M.Problem.from_arrays(nodes, faces, np.ones(len(faces), int), 1e-9, [[1], [-1]]))
    solver.solve_wavelength(om, ri, src, M.FP64, want_host=False)
    solver.shg_solve(om, ri, ri, [None, chi], M.FP64, want_host=False)  # `smed ... value`: the SH index is ri
    cs, ca = solver.cross_sections(2 * om, 1.0, [M.src_none()])
    assert abs(row[1] - cs[0]) <= 5e-4 * abs(cs[0]) and abs(row[2] - ca[0]) <= 5e-4 * abs(ca[0]), (row, cs, ca)
