"""The reference's own input: the example command script of its README on the
sphere mesh and gold refractive-index table it ships (data/sphere.msh,
data/aujc.ref), against the oracle's outputs in
tests/golden/reference_sphere_msh.npz (made by make_reference_input.py).

CPU: the product's Gmsh loader (mom_problem_load_gmsh) and the oracle's
restatement of load_mesh_gmsh read the reference's file identically to the
fixture (skipped where the reference checkout is absent), and the oracle's
get_refind reproduces the fixture's refractive indices.
GPU: the README script, run verbatim through the `mom` command interpreter on
the fixture's mesh and table written back as files (Gmsh 2.1 with three tags,
as in the reference's file), writes sphere-s1.crs rows that match the oracle
at four of the 100 wavelengths to the EN15.3 precision of the file; and the
same solve through the C ABI matches the oracle to 1e-9.
"""
import os
import subprocess

import numpy as np
import pytest

import mom_b200 as M
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "reference_sphere_msh.npz")
EXE = os.path.join(ROOT, "for90-mom2_b200", "bin", "mom_b200")
REF_MSH = "/root/reference/data/sphere.msh"
REF_TAB = "/root/reference/data/aujc.ref"

README_SCRIPT = """name 'sphere'
symm 1 id
mesh 'sphere.msh' 200d-9
wlrg 100 400d-9 1200d-9
nmed 2
smed 1 linear value (1.0, 0.0)
smed 2 linear file aujc.ref
ndom 2
sdom 1 1 15 0 1 -1
sdom 2 1 -15 0 2 -1
fdom
nsrc 1
ssrc 1 'pw' 0 90 0
solv
crst
exit
"""


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def write_inputs(d, g):
    """The fixture's mesh as a Gmsh 2.1 file with three tags per element
    (physical, elementary, partition) and its refractive-index table."""
    nodes, faces, ids = g["nodes"], g["faces"], g["ids"]
    with open(os.path.join(d, "sphere.msh"), "w") as fh:
        fh.write("$MeshFormat\n2.1 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(nodes))
        for i, p in enumerate(nodes):
            fh.write("%d %.17g %.17g %.17g\n" % (i + 1, p[0], p[1], p[2]))
        fh.write("$EndNodes\n$Elements\n%d\n" % len(faces))
        for i, (f, pid) in enumerate(zip(faces, ids)):
            fh.write("%d 2 3 %d 8 0 %d %d %d\n" % (i + 1, pid, f[0] + 1, f[1] + 1, f[2] + 1))
        fh.write("$EndElements\n")
    with open(os.path.join(d, "aujc.ref"), "w") as fh:
        for r in g["table"]:
            fh.write("  %.7e  %.7e  %.7e\n" % tuple(r))


@pytest.mark.skipif(not os.path.exists(REF_MSH), reason="reference checkout absent")
def test_loaders_read_the_reference_mesh(built, gold):
    n, f, i = O.load_mesh_gmsh(REF_MSH)
    assert np.array_equal(n, gold["nodes"]) and np.array_equal(f, gold["faces"]) and np.array_equal(i, gold["ids"])
    P = M.Problem.from_gmsh(REF_MSH, 200e-9, [[15], [-15]])
    Q = M.Problem.from_arrays(gold["nodes"], gold["faces"], gold["ids"], 200e-9, [[15], [-15]])
    assert P.nedges == Q.nedges == 4068
    for d in range(2):
        a, b = P.domain(d), Q.domain(d)
        for k in a:
            assert np.array_equal(a[k], b[k]), (d, k)


@pytest.mark.skipif(not os.path.exists(REF_TAB), reason="reference checkout absent")
def test_refractive_index_table(gold):
    for i, n in zip(gold["checked"], gold["ri"]):
        assert O.get_refind(REF_TAB, float(gold["wls"][i])) == n


def test_written_inputs_read_back(tmp_path, gold):
    write_inputs(str(tmp_path), gold)
    n, f, i = O.load_mesh_gmsh(str(tmp_path / "sphere.msh"))
    assert np.array_equal(n, gold["nodes"]) and np.array_equal(f, gold["faces"])
    for k, n_ref in zip(gold["checked"], gold["ri"]):
        assert O.get_refind(str(tmp_path / "aujc.ref"), float(gold["wls"][k])) == n_ref


@pytest.mark.gpu
def test_readme_script_matches_oracle(built, tmp_path, gold):
    write_inputs(str(tmp_path), gold)
    r = subprocess.run([EXE], input=README_SCRIPT, capture_output=True, text=True, cwd=tmp_path, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rows = [ln.split() for ln in open(tmp_path / "sphere-s1.crs") if ln.strip()]
    assert len(rows) == 100
    vals = np.array([[float(v) for v in row] for row in rows])
    for k, sca, ab in zip(gold["checked"], gold["csca"], gold["cabs"]):
        wl, csca, cabs = vals[k]
        assert abs(wl - gold["wls"][k]) <= 5e-4 * gold["wls"][k]
        # EN15.3: three decimals of a mantissa in [1, 1000)
        assert abs(csca - sca) <= 5e-4 * abs(sca), (k, csca, sca)
        assert abs(cabs - ab) <= 5e-4 * abs(ab), (k, cabs, ab)


@pytest.mark.gpu
def test_api_matches_oracle_at_full_precision(built, tmp_path, gold):
    write_inputs(str(tmp_path), gold)
    S = M.Solver(0)
    try:
        S.set_problem(M.Problem.from_gmsh(str(tmp_path / "sphere.msh"), 200e-9, [[15], [-15]]))
        src = [M.src_pw(0, 90, 0)]
        for k, n, sca, ab in zip(gold["checked"], gold["ri"], gold["csca"], gold["cabs"]):
            om = M.omega_of(float(gold["wls"][k]))
            S.solve_wavelength(om, [1.0, complex(n)], src, M.FP64, want_host=False)
            a, b = S.cross_sections(om, 1.0, src)
            assert abs(a[0] - sca) <= 1e-9 * abs(sca) and abs(b[0] - ab) <= 1e-9 * abs(ab), (k, a[0], sca, b[0], ab)
    finally:
        S.close()
