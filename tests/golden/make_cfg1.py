"""Regenerate tests/golden/oracle_sphere_s3.npz: the oracle's outputs at the
plain-FP64 single-solve configuration (icosphere s=3, r = 50 nm, 1280
triangles, 3840 unknowns, eps = -9 + 1.3i inside, vacuum outside, 600 nm,
x-polarised plane wave along +z), small enough to commit:
  blocks   relative Frobenius norms of the four PMCHWT blocks of A
  Av       A v for v = the seeded random vector below (the whole matrix,
           checked through one product)
  q, x     right-hand side and solution
  sigma    (sca, abs, ext)
  rcs      the 91 x 180 far field (rcst 1 1 91 180) every 5th theta, 9th phi,
           and its full-grid 2-norm
Run from the repository root:  python tests/golden/make_cfg1.py  (about a minute)
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "for90-mom2_b200")]
import oracle as O  # noqa: E402
from mom_b200 import meshgen  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def probe_vector(n):
    rng = np.random.default_rng(1234)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def main():
    nodes, faces = meshgen.icosphere(3, 50.0)
    ids = np.ones(len(faces), int)
    P = O.OracleProblem(nodes, faces, ids, 1e-9, [[1], [-1]])
    om = O.omega_of(600e-9)
    ri = [1.0 + 0j, complex(np.sqrt(-9 + 1.3j))]
    A = P.sysmat(om, ri)
    N = A.shape[0] // 2
    blocks = np.array([np.linalg.norm(A[:N, :N]), np.linalg.norm(A[N:, N:]), np.linalg.norm(A[N:, :N]),
                       np.linalg.norm(A[:N, N:])])
    v = probe_vector(2 * N)
    src = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)
    q = P.srcvec(om, ri[0], src)
    x = O.solve(A, q)
    sca, ab = P.cs(om, ri[0], x, src)
    rcs = P.rcs(om, ri[0], x, 91, 180)
    np.savez_compressed(os.path.join(HERE, "oracle_sphere_s3.npz"), blocks=blocks, Av=A @ v, q=q, x=x,
                        sigma=np.array([sca, ab, sca + ab]), rcs_sub=rcs[::5, ::9], rcs_norm=np.linalg.norm(rcs))


if __name__ == "__main__":
    main()
