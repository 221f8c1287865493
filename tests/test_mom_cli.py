"""The `mom` command interpreter (for90-mom2_b200/bin/mom_b200, the reference's
msgloop of interface.f90:1624-1734 over the C ABI).

CPU: command parsing, the set-up commands (mesh, ndom, sdom, fdom run on the
host) and the errors for input outside the linear PMCHWT path.  GPU: the
plain FP64 single-solve command script (icosphere s=3, 600 nm, x-polarised
plane wave) writes .crs and .rcs files whose EN15.3 values match the oracle's
committed cross sections and far field to the printed precision."""
import os
import subprocess

import numpy as np
import pytest

from mom_b200 import meshgen
from mom_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "for90-mom2_b200", "bin", "mom_b200")
GOLD = os.path.join(ROOT, "tests", "golden", "oracle_sphere_s3.npz")


def run(script, cwd):
    return subprocess.run([EXE], input=script, capture_output=True, text=True, cwd=cwd, timeout=600)


def setup_script(n_in):
    return "\n".join([
        "name 'sphere'",
        "symm 1 id",
        "mesh 'ico3.msh' 1d-9",
        "wlls 1 600d-9",
        "nmed 2",
        "smed 1 linear value (1.0, 0.0)",
        "smed 2 linear value (%.17g, %.17g)" % (n_in.real, n_in.imag),
        "ndom 2",
        "sdom 1 1 1 0 1 -1",
        "sdom 2 1 -1 0 2 -1",
        "fdom",
        "nsrc 1",
        "ssrc 1 'pw' 0 90 0",
    ]) + "\n"


@pytest.fixture(scope="module")
def workdir(built, tmp_path_factory):
    d = tmp_path_factory.mktemp("cli")
    nodes, faces, ids, _ = W.sphere(3)
    meshgen.write_gmsh22(str(d / "ico3.msh"), nodes, faces, ids)
    return d


def test_setup_commands_run_on_the_host(workdir):
    r = run(setup_script(np.sqrt(W.EPS_AU)) + "exit\n", workdir)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Allocated 2 media." in r.stdout and "Allocated 2 domains." in r.stdout
    assert "Allocated 1 sources." in r.stdout


def test_unknown_command_is_reported_and_skipped(workdir):
    r = run("frobnicate 1 2\nname x\nexit\n", workdir)
    assert r.returncode == 0 and "Unrecognized command frobnicate!" in r.stdout


@pytest.mark.parametrize("line,msg", [
    ("symm 1 r4", "rotation symmetry group 'r4'"),
    ("diff 1 1 0 0 false 0", "outside the linear PMCHWT path"),
])
def test_input_outside_the_path_stops(workdir, line, msg):
    r = run(line + "\nexit\n", workdir)
    assert r.returncode == 1 and msg in r.stdout


def test_mirror_groups_and_sbnd_are_accepted(workdir):
    """symm with mirror groups and sbnd run on the host (the reference's console lines)."""
    r = run("symm 3 mxp myp id\nmesh 'ico3.msh' 1d-9\nsbnd 7 xplane\nexit\n", workdir)
    assert r.returncode == 0, r.stdout
    assert "Created a symmetry group with 4 elements." in r.stdout
    assert "Classified 0 boundary edges" in r.stdout
    r = run("mesh 'ico3.msh' 1d-9\nsbnd 7 prdx1\nexit\n", workdir)
    assert r.returncode == 1 and "boundary type 'prdx1'" in r.stdout


def test_periodic_green_function_stops(workdir):
    script = setup_script(2.0).replace("sdom 2 1 -1 0 2 -1", "sdom 2 1 -1 0 2 1")
    r = run(script + "exit\n", workdir)
    assert r.returncode == 1 and "periodic Green's functions" in r.stdout


def test_missing_mesh_file_stops(workdir):
    r = run("mesh 'nothere.msh' 1d-9\nexit\n", workdir)
    assert r.returncode == 1 and "mesh nothere.msh" in r.stdout


def read_en(path):
    rows = [l.split() for l in open(path) if l.strip()]
    return np.array([[float(v) for v in r] for r in rows]), rows


def half_ulp(token):
    """Half a unit in the last printed place of an EN15.3 field."""
    return 0.5e-3 * 10.0 ** int(token.split("E")[1])


@pytest.mark.gpu
def test_fp64_command_script_matches_oracle(workdir):
    ref = np.load(GOLD)
    script = setup_script(np.sqrt(W.EPS_AU)) + ("solv\ncrst\nrcst 1 1 91 180\n"
                                                "nfpl 1 1 -100d-9 0 -100d-9 200d-9 0 0 0 0 200d-9 5 4 'xz'\nexit\n")
    r = run(script, workdir)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    crs, tok = read_en(workdir / "sphere-s1.crs")
    assert crs.shape == (1, 3)
    assert abs(crs[0, 0] - 600e-9) <= float(half_ulp(tok[0][0]))
    for j, k in ((1, 0), (2, 1)):  # csca, cabs against the oracle (sigma = [csca, cabs, cext])
        assert abs(crs[0, j] - ref["sigma"][k]) <= half_ulp(tok[0][j]) * 1.001 + 1e-9 * abs(ref["sigma"][k])
    rcs, tok = read_en(workdir / "sphere-wl1-s1.rcs")
    assert rcs.shape == (91, 180)
    sub = rcs[::5, ::9]
    tol = np.array([[half_ulp(t) for t in row[::9]] for row in tok[::5]])
    assert np.all(np.abs(sub - ref["rcs_sub"]) <= tol * 1.001 + 1e-9 * np.abs(ref["rcs_sub"]))
    # nfpl: total field (scattered + incident) of domain 1 on a 5 x 4 grid in the
    # xz plane, in the basis (x, z, x cross z = -y), against the library's
    # scat_fields on the same FP64 solution
    import mom_b200 as M
    nodes, faces, ids, doms = W.sphere(3)
    S = M.Solver(0)
    try:
        S.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, doms))
        om, src = M.omega_of(600e-9), M.src_pw(0, 90, 0)
        x = S.solve_wavelength(om, [1.0, np.sqrt(W.EPS_AU)], [src], M.FP64, 1e-12, 30)
        a, b = np.meshgrid(np.arange(5), np.arange(4), indexing="ij")
        pts = np.stack([-100e-9 + a.ravel() / 4 * 200e-9, 0 * a.ravel(), -100e-9 + b.ravel() / 3 * 200e-9], axis=1)
        e, h = S.scat_fields(om, 1.0, pts, x=x, srcs=[src], dom=0)
    finally:
        S.close()
    basis = np.array([[1, 0, 0], [0, 0, 1], [0, -1, 0]], dtype=float)
    for name, f in (("e", e[0]), ("h", h[0])):
        loc = f @ basis.T  # [npts][3] in the plane basis
        for c, comp in enumerate("xyz"):
            for part, fn in (("re", np.real), ("im", np.imag)):
                vals, tok = read_en(workdir / ("sphere-wl1-s1-d1-xz-%s%s-%s.dat" % (name, comp, part)))
                assert vals.shape == (4, 5)
                want = fn(loc[:, c]).reshape(5, 4).T
                tol = np.array([[half_ulp(t) for t in row] for row in tok])
                assert np.all(np.abs(vals - want) <= tol * 1.001 + 1e-9 * np.abs(want).max())


def test_en15_3_output_format(tmp_path):
    """write_data's EN15.3 fields (aux.f90:192-211): engineering notation, three
    decimals, 15 columns; checked by compiling the interpreter's formatter alone."""
    import shutil
    if not shutil.which("g++"):
        pytest.skip("no host C++ compiler")
    src = tmp_path / "en.cpp"
    src.write_text(
        '#define main mom_main_unused\n#include "%s"\n#undef main\n'
        'int main() { const double v[] = {6e-7, 0.0, -3.5e-16, 999.9996, 12345.6789, 1.0, 9.9999996e-10};\n'
        '  for (double x : v) std::printf("[%%s]\\n", en15_3(x).c_str()); }\n'
        % os.path.join(ROOT, "for90-mom2_b200", "host", "mom_main.cpp"))
    exe = tmp_path / "en"
    subprocess.run(["g++", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-o", str(exe), str(src),
                    "-L" + os.path.join(ROOT, "for90-mom2_b200", "lib"), "-lmomgpu",
                    "-Wl,-rpath," + os.path.join(ROOT, "for90-mom2_b200", "lib")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()
    assert out == ["[    600.000E-09]", "[      0.000E+00]", "[   -350.000E-18]", "[      1.000E+03]",
                   "[     12.346E+03]", "[      1.000E+00]", "[      1.000E-09]"]
