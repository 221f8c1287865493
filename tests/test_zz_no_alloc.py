"""Allocation-free cross sections (mom_gpu_cross_sections_noalloc), through the C ABI.

Callers whose device memory is reserved up front by another allocator, or
that cannot accept the device-wide synchronisation of cudaMalloc/cudaFree,
use this entry point: it keeps its scratch in a fixed array inside the
library.  It must give the same cross sections as the allocating entry point
(mom_gpu_cross_sections) on the same device solutions, call after call.
This file is collected last so that a stop at the first failure has already
run every other test.
"""
import numpy as np
import pytest

import mom_b200 as M
from mom_b200 import meshgen

pytestmark = pytest.mark.gpu


def test_noalloc_cross_sections_match_allocating_entry_point(built):
    S = M.Solver(0)
    try:
        nodes, faces = meshgen.icosphere(2, 50.0)
        ids = np.ones(len(faces), dtype=np.int32)
        S.set_problem(M.Problem.from_arrays(nodes, faces, ids, 1e-9, [[1], [-1]]))
        om = M.omega_of(600e-9)
        ri = [1.0, np.sqrt(-9 + 1.3j)]
        srcs = [M.src_pw(0, 90, 0), M.src_pw(90, 0, 30), M.src_pw_elliptic(30, 40, np.exp(0.7j))]
        S.solve_wavelength(om, ri, srcs, precision=M.FP64)
        ref_sca, ref_abs = S.cross_sections(om, ri[0], srcs)
        x_dev, ldx, ns = S.device_solution()
        assert ns == len(srcs) and x_dev
        for _ in range(2):  # two calls in a row share the scratch array
            sca, ab = S.cross_sections_noalloc(om, ri[0], srcs, x_dev, ldx)
            np.testing.assert_allclose(sca, ref_sca, rtol=1e-12, atol=0)
            np.testing.assert_allclose(ab, ref_abs, rtol=1e-12, atol=0)
        # after the warm-up calls above, further calls leave the device's free
        # memory unchanged (nothing is allocated per call)
        import torch
        torch.cuda.synchronize(0)
        free0 = torch.cuda.mem_get_info(0)[0]
        for _ in range(3):
            sca, ab = S.cross_sections_noalloc(om, ri[0], srcs, x_dev, ldx)
        torch.cuda.synchronize(0)
        assert torch.cuda.mem_get_info(0)[0] == free0
        np.testing.assert_allclose(sca, ref_sca, rtol=1e-12, atol=0)
        # a request beyond the fixed scratch size is rejected, not truncated
        with pytest.raises(M.MomError) as err:
            S.cross_sections_noalloc(om, ri[0], [srcs[0]] * 65, x_dev, ldx)
        assert err.value.status == M.MOM_ERR_ARG
        # so is a leading dimension shorter than the 2N unknowns
        with pytest.raises(M.MomError) as err:
            S.cross_sections_noalloc(om, ri[0], srcs, x_dev, 2 * S.N - 1)
        assert err.value.status == M.MOM_ERR_ARG
    finally:
        S.close()
