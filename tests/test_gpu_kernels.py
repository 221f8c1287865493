"""GPU unit tests of individual kernels (through the C ABI)."""
import numpy as np
import pytest

import mom_b200 as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver(built):
    s = M.Solver(0)
    yield s
    s.close()


@pytest.mark.parametrize("m,nc,k", [(64, 100, 256), (320, 600, 64), (128, 256, 256), (192, 513, 128), (64, 64, 64),
                                    (1984, 192, 64)])
def test_tensor_core_update_matches_fp64(solver, m, nc, k):
    """The LU trailing update C -= L U on tcgen05 (3xTF32) is FP32-accurate:
    relative Frobenius error <= 1e-5 against the FP64 product of the same FP32
    inputs (a single TF32 pass would give ~1e-3)."""
    rng = np.random.default_rng(m + nc + k)
    cplx = lambda r, c: (rng.standard_normal((r, c)) + 1j * rng.standard_normal((r, c))).astype(np.complex64)
    L, U, C = cplx(m, k), cplx(k, nc), cplx(m, nc)
    out = solver.selftest_cgemm(L, U, C)
    ref = C.astype(np.complex128) - L.astype(np.complex128) @ U.astype(np.complex128)
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert err <= 1e-5, err
