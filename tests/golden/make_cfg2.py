"""Regenerate tests/golden/oracle_sphere_s4.npz: the oracle's FP64 outputs at
the mixed-precision-at-scale configuration (icosphere s=4, r = 50 nm, 5120
triangles, 15,360 unknowns, eps = -9 + 1.3i inside, vacuum outside, 600 nm,
x-polarised plane wave along +z):
  blocks   Frobenius norms of the four PMCHWT blocks of A
  Av       A v for v = the seeded random vector of probe_vector (the whole
           matrix, checked through one product)
  q, x     right-hand side and solution (ZGETRF + ZGETRS)
  sigma    (sca, abs, ext)
  berr     backward error ||A x - q|| / (||A||_F ||x||) of the oracle solve
Run from the repository root:  python tests/golden/make_cfg2.py
(about 5 minutes of assembly on 8 cores, 10 GB of host memory).
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "for90-mom2_b200")]
import oracle as O  # noqa: E402
from mom_b200 import meshgen  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def probe_vector(n):
    rng = np.random.default_rng(4321)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def main():
    t0 = time.time()
    nodes, faces = meshgen.icosphere(4, 50.0)
    ids = np.ones(len(faces), int)
    P = O.OracleProblem(nodes, faces, ids, 1e-9, [[1], [-1]])
    om = O.omega_of(600e-9)
    ri = [1.0 + 0j, complex(np.sqrt(-9 + 1.3j))]
    A = P.sysmat(om, ri)
    print("sysmat %.1f s" % (time.time() - t0), flush=True)
    N = A.shape[0] // 2
    blocks = np.array([np.linalg.norm(A[:N, :N]), np.linalg.norm(A[N:, N:]), np.linalg.norm(A[N:, :N]),
                       np.linalg.norm(A[:N, N:])])
    v = probe_vector(2 * N)
    Av = A @ v
    src = dict(type="pw", theta=0.0, phi=90 * O.DEGTORAD, psi=0.0)
    q = P.srcvec(om, ri[0], src)
    x = O.solve(A, q)
    print("solve %.1f s" % (time.time() - t0), flush=True)
    berr = np.linalg.norm(A @ x - q) / (np.linalg.norm(A) * np.linalg.norm(x))
    sca, ab = P.cs(om, ri[0], x, src)
    np.savez_compressed(os.path.join(HERE, "oracle_sphere_s4.npz"), blocks=blocks, Av=Av, q=q, x=x,
                        sigma=np.array([sca, ab, sca + ab]), berr=np.array(berr))
    print("sigma sca %.12e abs %.12e ext %.12e, backward error %.2e, %.1f s" % (sca, ab, sca + ab, berr,
                                                                               time.time() - t0))


if __name__ == "__main__":
    main()
