"""Regenerate tests/golden/reference_sphere_msh.npz from the reference's own
input data: the example command script of the reference's README (a sphere
of radius 200 nm from data/sphere.msh, physical surface 15, 100 wavelengths
on 400-1200 nm, exterior vacuum, interior gold from the refractive-index
table data/aujc.ref, x-polarised plane wave along +z, crst), run through the
oracle at four of its wavelengths.

The mesh is read by the oracle's restatement of load_mesh_gmsh and the
refractive indices by its restatement of get_refind (single-precision
rounding kept).  Stored: the mesh as arrays (nodes, faces, physical ids),
the refractive-index table, the wavelengths of `wlrg 100 400d-9 1200d-9`,
the indices of the four checked wavelengths, the oracle's refractive index
there and its sigma_sca, sigma_abs.  The GPU test writes the mesh and the
table back as files and runs the README script through the `mom` command
interpreter; it never reads the reference tree.

Run from the repository root:  python tests/golden/make_reference_input.py
(about 5 minutes on 8 cores; needs the reference checkout).
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle")]
import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DATA = "/root/reference/data"
CHECKED = [0, 33, 66, 99]


def main():
    t0 = time.time()
    msh = os.path.join(REF_DATA, "sphere.msh")
    tab = os.path.join(REF_DATA, "aujc.ref")
    nodes, faces, ids = O.load_mesh_gmsh(msh)
    table = np.loadtxt(tab)
    wls = np.array([400e-9 + (i / 99.0) * (1200e-9 - 400e-9) for i in range(100)])
    P = O.OracleProblem(nodes, faces, ids, 200e-9, [[15], [-15]])
    src = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)
    ri, sca, ab = [], [], []
    for i in CHECKED:
        wl = float(wls[i])
        n = O.get_refind(tab, wl)
        om = O.omega_of(wl)
        r = [1.0 + 0j, n]
        A = P.sysmat(om, r)
        q = P.srcvec(om, r[0], src)
        x = O.solve(A, q)
        s1, s2 = P.cs(om, r[0], x, src)
        ri.append(n)
        sca.append(s1)
        ab.append(s2)
        print("wl %.6e n %s sca %.12e abs %.12e (%.0f s)" % (wl, n, s1, s2, time.time() - t0), flush=True)
    np.savez_compressed(os.path.join(HERE, "reference_sphere_msh.npz"), nodes=nodes, faces=faces, ids=ids,
                        table=table, wls=wls, checked=np.array(CHECKED), ri=np.array(ri), csca=np.array(sca),
                        cabs=np.array(ab))


if __name__ == "__main__":
    main()
