"""Regenerate tests/golden/adjoint_fd_s1.json: central finite differences of the
oracle's (the CPU restatement's) cross sections on a radially perturbed
1-subdivision sphere, the reference the adjoint gradients are checked
against.  Steps: 1e-6 in eps (real and imaginary part), 1e-4 nm in vertex
coordinates.  Run from the repository root:
    python tests/golden/make_adjoint_fd.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "for90-mom2_b200")]
import oracle as O  # noqa: E402
from mom_b200 import meshgen  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
WL = 600e-9
EPS = -9 + 1.3j
SRC = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)


def sigma(nodes, faces, eps):
    ids = np.ones(len(faces), int)
    P = O.OracleProblem(nodes, faces, ids, 1e-9, [[1], [-1]])
    ri = [1.0 + 0j, complex(np.sqrt(eps))]
    om = O.omega_of(WL)
    x = O.solve(P.sysmat(om, ri), P.srcvec(om, ri[0], SRC))
    sca, ab = P.cs(om, ri[0], x, SRC)
    return np.array([sca + ab, ab])


def main():
    nodes, faces = meshgen.perturbed_sphere(1, 50.0, lmax=4, sigma=0.03, seed=4)
    s0 = sigma(nodes, faces, EPS)
    h = 1e-6
    deps = []
    for dz in (h, 1j * h):
        deps.append(((sigma(nodes, faces, EPS + dz) - sigma(nodes, faces, EPS - dz)) / (2 * h)).tolist())
    rng = np.random.default_rng(11)
    picks = [(int(v), int(k)) for v, k in zip(rng.choice(len(nodes), 8, replace=False), rng.integers(0, 3, 8))]
    hv = 1e-4
    dverts = []
    for v, k in picks:
        npl, nmi = nodes.copy(), nodes.copy()
        npl[v, k] += hv
        nmi[v, k] -= hv
        fd = (sigma(npl, faces, EPS) - sigma(nmi, faces, EPS)) / (2 * hv)
        dverts.append([v, k, fd.tolist()])
    out = dict(mesh="perturbed sphere s=1 r=50 nm (lmax 4, sigma 0.03, seed 4), domains [[1],[-1]], tri_gl13",
               wavelength=WL, eps=[EPS.real, EPS.imag], source="pw theta=0 phi=90 psi=0",
               sigma=s0.tolist(), deps_step=h, vertex_step_nm=hv,
               deps=deps,  # [Re, Im][ext, abs]
               dverts=dverts)  # (vertex, coordinate, [ext, abs] per nm)
    with open(os.path.join(HERE, "adjoint_fd_s1.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()
