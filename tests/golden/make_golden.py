"""Regenerate tests/golden/oracle_sphere_s1.json (the oracle's own output on a
1-subdivision icosphere; a regression pin for the CPU restatement) and the
Mie reference values.  Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "for90-mom2_b200")]
import oracle as O  # noqa: E402
import mie  # noqa: E402
from mom_b200 import meshgen  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    nodes, faces = meshgen.icosphere(1, 50.0)
    ids = np.ones(len(faces), int)
    P = O.OracleProblem(nodes, faces, ids, 1e-9, [[1], [-1]])
    wl = 600e-9
    ri = [1.0 + 0j, complex(np.sqrt(-9 + 1.3j))]
    om = O.omega_of(wl)
    A = P.sysmat(om, ri)
    rng = np.random.default_rng(0)
    picks = [(int(i), int(j)) for i, j in rng.integers(0, A.shape[0], size=(12, 2))]
    src = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)
    x = O.solve(A, P.srcvec(om, ri[0], src))
    sca, ab = P.cs(om, ri[0], x, src)
    out = dict(mesh="icosphere s=1 r=50 nm (80 faces, 240 unknowns), domains [[1],[-1]], tri_gl13",
               wavelength=wl, ri=[[v.real, v.imag] for v in ri], A_frobenius=float(np.linalg.norm(A)),
               A_entries=[[i, j, float(A[i, j].real), float(A[i, j].imag)] for i, j in picks],
               csca=sca, cabs=ab, mie=list(mie.mie_cross_sections(50e-9, wl, ri[1])))
    with open(os.path.join(HERE, "oracle_sphere_s1.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()
