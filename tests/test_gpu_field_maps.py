"""Field maps on meshes and volumes: the surface fields of field_mesh (nfms)
through mom_gpu_surface_fields against the oracle's restatement, with and
without a symmetry group, and the interpreter's nfms / nfem / nfdm commands
(Gmsh post-processing files of save_vector_fields_msh and
save_domain_vector_fields_msh) against the C ABI.

Tolerances: surface fields 1e-12 relative to the oracle (FP64, the same
currents); the eighth sphere's image faces against the full sphere's faces
1e-9 (s=1: the same discretisation); file values to the EN15.3 precision."""
import os
import subprocess

import numpy as np
import pytest

import mom_b200 as M
import oracle as O
from mom_b200 import meshgen
from mom_b200 import workloads as W

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "for90-mom2_b200", "bin", "mom_b200")
WL = 600e-9


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def solver(built):
    s = M.Solver(0)
    yield s
    s.close()


def test_surface_fields_match_oracle(solver):
    nodes, faces, ids, doms = W.sphere(2)
    P = O.OracleProblem(nodes, faces, ids, 1e-9, doms)
    om = M.omega_of(WL)
    n_in = np.sqrt(W.EPS_AU)
    srcs = [M.src_pw(0, 90, 0), M.src_pw_elliptic(35, 20, np.exp(0.4j))]
    osrc = [dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0),
            dict(type="pw_elliptic", theta=35 * O.DEGTORAD, phi=20 * O.DEGTORAD, phase=np.exp(0.4j))]
    A = P.sysmat(om, np.array([1.0, n_in]))
    x = O.solve(A, np.stack([P.srcvec(om, 1.0, s) for s in osrc], axis=1))
    solver.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    for d, ri in ((0, 1.0), (1, n_in)):
        for k in range(2):
            e, h = solver.surface_fields(om, ri, isrc=k, x=x, dom=d)
            eo, ho = O.field_mesh(P, d, om, complex(ri), x[:, k])
            assert rel(e, eo) <= 1e-12 and rel(h, ho) <= 1e-12, (d, k, rel(e, eo), rel(h, ho))
    # device solutions: the same as the host ones after a GPU solve of the same system
    solver.solve_wavelength(om, [1.0, n_in], srcs, M.FP64, want_host=False)
    e, h = solver.surface_fields(om, 1.0, isrc=1, dom=0)
    eo, ho = O.field_mesh(P, 0, om, 1.0, x[:, 1])
    assert rel(e, eo) <= 1e-9 and rel(h, ho) <= 1e-9


def test_surface_fields_with_group_match_full_sphere(solver):
    """The eighth of the s=1 octahedron sphere with mxp x myp x mzp: the fields on
    all 8 images of its faces equal the full sphere's fields on the same faces."""
    nodes, faces = meshgen.octasphere(1, 50.0)
    om = M.omega_of(WL)
    ri = [1.0, np.sqrt(complex(-9, 1.3))]
    src = [M.src_pw(17, 40, 25)]
    solver.set_problem(M.Problem.from_arrays(nodes, faces, np.ones(len(faces), int), 1e-9, [[1], [-1]]))
    solver.solve_wavelength(om, ri, src, M.FP64, want_host=False)
    e_full, h_full = solver.surface_fields(om, ri[0], dom=0)
    cp_full = (nodes[faces].mean(axis=1)) * 1e-9
    fn, ff, lines = meshgen.symmetry_fragment(nodes, faces, [0, 1, 2])
    prob = M.Problem.from_arrays(fn, ff, np.ones(len(ff), int), 1e-9, [[1], [-1]])
    prob.set_lines(np.concatenate([np.asarray(lines[ax], np.int32).reshape(-1, 2) for ax in range(3)]),
                   np.concatenate([np.full(len(lines[ax]), 10 + ax, np.int32) for ax in range(3)]))
    for ax, nm in enumerate(("xplane", "yplane", "zplane")):
        prob.classify_edges(10 + ax, nm)
    solver.set_problem(prob)
    nga = solver.set_symmetry(["mxp", "myp", "mzp"], prob)
    solver.solve_wavelength(om, ri, src, M.FP64, want_host=False)
    e, h = solver.surface_fields(om, ri[0], dom=0)
    cp = fn[ff].mean(axis=1) * 1e-9
    F = len(ff)
    for g in range(nga):
        J, _ = solver.group_action(g)
        for f in range(F):
            c = J @ cp[f]
            i = int(np.argmin(np.linalg.norm(cp_full - c, axis=1)))
            assert np.linalg.norm(cp_full[i] - c) < 1e-15
            assert np.linalg.norm(e[g * F + f] - e_full[i]) <= 1e-9 * np.linalg.norm(e_full[i]), (g, f)
            assert np.linalg.norm(h[g * F + f] - h_full[i]) <= 1e-9 * np.linalg.norm(h_full[i]), (g, f)


def read_msh_blocks(path):
    """(nodes, elements, data) of a Gmsh 2.1 post-processing file: data maps
    (section, name, time step) to {entity index: values}."""
    lines = open(path).read().split("\n")
    nodes, elems, data = {}, {}, {}
    i = 0
    while i < len(lines):
        t = lines[i].strip()
        if t == "$Nodes":
            n = int(lines[i + 1])
            for ln in lines[i + 2:i + 2 + n]:
                p = ln.split()
                nodes[int(p[0])] = [float(v) for v in p[1:4]]
            i += n + 3
        elif t == "$Elements":
            n = int(lines[i + 1])
            for ln in lines[i + 2:i + 2 + n]:
                p = ln.split()
                elems[int(p[0])] = [int(v) for v in p[1:]]
            i += n + 3
        elif t in ("$ElementData", "$NodeData"):
            name = lines[i + 2].strip().strip('"')
            step = int(lines[i + 5])
            ncomp = int(lines[i + 6])
            n = int(lines[i + 7])
            vals = {}
            for ln in lines[i + 8:i + 8 + n]:
                p = ln.split()
                vals[int(p[0])] = [float(v) for v in p[1:1 + ncomp]]
            data[(t, name, step)] = vals
            i += n + 9
        else:
            i += 1
    return nodes, elems, data


def close_en(a, b):
    """Agreement to the EN15.3 precision (3 decimals of a mantissa in [1, 1000))."""
    a, b = np.asarray(a), np.asarray(b)
    return np.all(np.abs(a - b) <= 5e-4 * np.maximum(np.abs(b), 1e-3 * np.abs(b).max()) + 1e-30)


def test_field_map_commands(solver, tmp_path):
    nodes, faces, ids, doms = W.sphere(2)
    meshgen.write_gmsh22(str(tmp_path / "ico2.msh"), nodes, faces, ids)
    en, ef = meshgen.icosphere(1, 80.0)
    meshgen.write_gmsh22(str(tmp_path / "ext.msh"), en, ef, np.ones(len(ef), int))
    n_in = np.sqrt(W.EPS_AU)
    script = "\n".join([
        "name 'maps'", "symm 1 id", "mesh 'ico2.msh' 1d-9", "wlls 1 600d-9", "nmed 2",
        "smed 1 linear value (1.0, 0.0)", "smed 2 linear value (%.17g, %.17g)" % (n_in.real, n_in.imag),
        "ndom 2", "sdom 1 1 1 0 1 -1", "sdom 2 1 -1 0 2 -1", "fdom", "nsrc 1", "ssrc 1 'pw' 0 90 0",
        "solv", "nfms 1 1 1", "nfem 1 1 1 'ext.msh' true", "nfdm 1 1 1 true 0 0 0 200d-9 200d-9 200d-9 5 4 3",
        "exit"]) + "\n"
    # nfms, nfem and nfdm write the same file name in turn: run the script up to
    # each command alone
    nfem_cmd = "nfem 1 1 1 'ext.msh' true\n"
    nfdm_cmd = "nfdm 1 1 1 true 0 0 0 200d-9 200d-9 200d-9 5 4 3\n"
    r = subprocess.run([EXE], input=script.replace(nfem_cmd, "").replace(nfdm_cmd, ""), capture_output=True,
                       text=True, cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:]
    om = M.omega_of(WL)
    solver.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
    src = [M.src_pw(0, 90, 0)]
    solver.solve_wavelength(om, [1.0, n_in], src, M.FP64, want_host=False)
    path = tmp_path / "maps-wl1-s1-d1.msh"
    # nfms: frame 25 (step 24) of Re(E) is Re(E) itself
    e, h = solver.surface_fields(om, 1.0, dom=0)
    nd, el, data = read_msh_blocks(path)
    assert len(el) == len(faces) and len(nd) == len(nodes)
    got = np.array([data[("$ElementData", "Re(E)", 24)][i + 1] for i in range(len(faces))])
    assert close_en(got, e.real)
    got = np.array([data[("$ElementData", "Re(H)", 24)][i + 1] for i in range(len(faces))])
    assert close_en(got, h.real)
    assert len([k for k in data if k[1] == "|Re(E)|"]) == 25
    for cmd in ("nfem", "nfdm"):
        sc = script.replace("nfms 1 1 1\n", "").replace(nfem_cmd if cmd == "nfdm" else nfdm_cmd, "")
        r = subprocess.run([EXE], input=sc, capture_output=True, text=True, cwd=tmp_path, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:]
        nd, el, data = read_msh_blocks(path)
        if cmd == "nfem":
            cp = (en[ef].mean(axis=1)) * 1e-9
            ee, hh = solver.scat_fields(om, 1.0, cp, srcs=src, dom=0)
            assert len(el) == len(ef)
            got = np.array([data[("$ElementData", "Re(E)", 24)][i + 1] for i in range(len(ef))])
            assert close_en(got, ee[0].real)
        else:
            g = [np.float32(np.arange(k)) / np.float32(k - 1) for k in (5, 4, 3)]
            pts = np.array([[-100e-9 + 200e-9 * float(a), -100e-9 + 200e-9 * float(b), -100e-9 + 200e-9 * float(c)]
                            for a in g[0] for b in g[1] for c in g[2]])
            ee, hh = solver.scat_fields(om, 1.0, pts, srcs=src, dom=0)
            mag = np.linalg.norm(ee[0], axis=1)
            keep = np.nonzero(mag > 0.01 * mag.max())[0]
            nn = len(nodes)
            assert len(nd) == nn + len(keep) and len(el) == len(faces) + len(keep)
            vals = data[("$NodeData", "Re(E)", 24)]
            got = np.array([vals[nn + i + 1] for i in range(len(keep))])
            assert close_en(got, ee[0][keep].real)
