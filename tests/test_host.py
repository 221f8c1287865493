"""CPU tests of the product's host side: problem set-up (mesh / sdom / fdom),
the C ABI surface of libmomgpu.so, error codes, and bench.py's CPU arms."""
import ctypes
import json
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import mom_b200 as M
import oracle as O
from mom_b200 import meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def core_shell(s):
    n1, f1 = meshgen.icosphere(s, 40.0)
    n2, f2 = meshgen.icosphere(s, 60.0)
    nodes = np.vstack([n1, n2])
    faces = np.vstack([f1, f2 + len(n1)])
    ids = np.r_[np.full(len(f1), 1), np.full(len(f2), 2)]
    return nodes, faces, ids, [[2], [-2, 1], [-1]]


CASES = {
    "sphere1": lambda: (*meshgen.icosphere(1, 50.0), None, [[1], [-1]]),
    "sphere3": lambda: (*meshgen.icosphere(3, 50.0), None, [[1], [-1]]),
    "coreshell2": lambda: core_shell(2),
}


@pytest.mark.parametrize("name", list(CASES))
def test_topology_matches_oracle(built, name):
    """build_mesh / extract_submesh / invert_faces / submesh_edge_connectivity /
    orient_basis: the product's O(F) C++ set-up reproduces the reference
    algorithm (restated literally in the oracle) bit for bit."""
    nodes, faces, ids, doms = CASES[name]()
    if ids is None:
        ids = np.ones(len(faces), int)
    P = O.OracleProblem(nodes, faces, ids, 1e-9, doms)
    Q = M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms)
    assert Q.nedges == P.N and Q.ndom == len(doms)
    for d in [-1] + list(range(len(doms))):
        a, b = P.export(d), Q.domain(d)
        for k in ("face_node", "face_edge", "edge_node", "edge_face", "edge_bnode"):
            assert np.array_equal(a[k], b[k]), (d, k)
        assert np.array_equal(a["nodes"], b["nodes"])
        if d >= 0:
            assert np.array_equal(a["edge_parent"], b["edge_parent"])


def test_gmsh_roundtrip(built, tmp_path):
    nodes, faces, ids, doms = core_shell(1)
    path = str(tmp_path / "cs.msh")
    meshgen.write_gmsh22(path, nodes, faces, ids)
    A = M.Problem.from_gmsh(path, 1e-9, doms)
    B = M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms)
    for d in range(3):
        a, b = A.domain(d), B.domain(d)
        for k in a:
            assert np.array_equal(a[k], b[k])


def test_every_declared_entry_point_is_exported(built):
    hdr = open(os.path.join(ROOT, "include", "mom_gpu.h")).read()
    names = sorted(set(re.findall(r"\b(mom_(?:gpu|problem|tri)_\w+)\s*\(", hdr)))
    assert len(names) >= 30
    lib = M.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(M.EXPORTS) <= set(names)


def test_triangle_rules_match_oracle(built):
    for name in ("tri_gl1", "tri_gl3", "tri_gl4", "tri_gl7", "tri_gl13"):
        w, nd = M.tri_rule(name)
        wo, ndo = O.tri_rule(name)
        assert np.array_equal(w, wo) and np.array_equal(nd, ndo), name
    with pytest.raises(M.MomError):
        M.tri_rule("tri_gl5")


def test_problem_errors(built):
    nodes, faces = meshgen.icosphere(1, 50.0)
    ids = np.ones(len(faces), int)
    with pytest.raises(M.MomError) as e:  # zero is not a valid surface id (interface.f90:80-83)
        M.Problem.from_arrays(nodes, faces, ids, 1e-9, [[1], [0]])
    assert e.value.status == M.MOM_ERR_ARG
    with pytest.raises(M.MomError) as e:  # every edge needs two children (mesh.f90:415-418)
        M.Problem.from_arrays(nodes, faces, ids, 1e-9, [[1]])
    assert e.value.status == M.MOM_ERR_MESH
    with pytest.raises(M.MomError) as e:
        M.Problem.from_gmsh("/nonexistent/file.msh", 1e-9, [[1], [-1]])
    assert e.value.status == M.MOM_ERR_IO


def test_strerror_and_no_device(built):
    L = M.lib()
    assert L.mom_gpu_strerror(M.MOM_ERR_SINGULAR).decode().startswith("Matrix factorization failed")
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        h = ctypes.c_void_p()
        assert L.mom_gpu_create(0, ctypes.byref(h)) == M.MOM_ERR_CUDA and not h.value


def test_bench_reference_arm_json():
    """bench.py --impl reference: the CPU arm (oracle + OpenBLAS) prints one JSON line."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--subdiv", "1",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "solves/s"
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0


def test_sbnd_classifies_plane_edges(built, tmp_path):
    """sbnd / classify_edges on the host: line elements read from a Gmsh file
    (type 1, physical id as the first tag) mark the master edges they cover;
    edges elsewhere stay MOM_BND_NONE."""
    nodes, faces = meshgen.octasphere(2, 50.0)
    fn, ff, lines = meshgen.symmetry_fragment(nodes, faces, [0, 1])
    path = tmp_path / "quarter.msh"
    with open(path, "w") as fh:
        fh.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(fn))
        for i, p in enumerate(fn):
            fh.write("%d %.17g %.17g %.17g\n" % (i + 1, p[0], p[1], p[2]))
        ne = len(lines[0]) + len(lines[1]) + len(ff)
        fh.write("$EndNodes\n$Elements\n%d\n" % ne)
        k = 1
        for ax, pid in ((0, 21), (1, 22)):
            for a, b in lines[ax]:
                fh.write("%d 1 2 %d %d %d %d\n" % (k, pid, pid, a + 1, b + 1))
                k += 1
        for f in ff:
            fh.write("%d 2 2 1 1 %d %d %d\n" % (k, f[0] + 1, f[1] + 1, f[2] + 1))
            k += 1
        fh.write("$EndElements\n")
    P = M.Problem.from_gmsh(str(path), 1e-9, [[1], [-1]])
    assert P.classify_edges(21, "xplane") == len(lines[0])
    assert P.classify_edges(22, "yplane") == len(lines[1])
    assert P.classify_edges(99, "zplane") == 0
    bnd = P.edge_bnd()
    assert np.count_nonzero(bnd == M.BND_XPLANE) == len(lines[0])
    assert np.count_nonzero(bnd == M.BND_YPLANE) == len(lines[1])
    assert np.count_nonzero(bnd == M.BND_NONE) == len(bnd) - len(lines[0]) - len(lines[1])
    # the same through line arrays
    Q = M.Problem.from_arrays(fn, ff, np.ones(len(ff), int), 1e-9, [[1], [-1]])
    Q.set_lines(np.asarray(lines[0]), 21)
    assert Q.classify_edges(21, M.BND_XPLANE) == len(lines[0])
    assert np.array_equal(Q.edge_bnd() == M.BND_XPLANE, bnd == M.BND_XPLANE)
