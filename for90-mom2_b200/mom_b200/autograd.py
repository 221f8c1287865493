"""torch.autograd wrapper of the adjoint entry point, for gradient checks.

``cross_sections(solver, eps_re, eps_im, nodes_nm, faces, face_ids, domains,
eps_dom, omega, ri, src, precision)`` returns a float64 tensor
[sigma_ext, sigma_abs] of one plane-wave source and differentiates it with
respect to the permittivity eps = eps_re + i eps_im of interior domain
``eps_dom`` and the master-mesh node coordinates (nm).  Forward: set the
problem, solve (mom_gpu_solve_wavelength) and cs_prtsrf
(mom_gpu_cross_sections).  Backward: the gradients of one call of
mom_gpu_adjoint (one transposed solve on the same LU factors, the
face-pair derivatives recomputed on the GPU), taken in forward and scaled by
the incoming gradient.  The solve itself runs in the library; torch only
carries the numbers, so this is a thin harness, not a compute path.
"""
from __future__ import annotations

import numpy as np
import torch

from . import Problem


class CrossSectionsFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eps_re, eps_im, nodes_nm, solver, faces, face_ids, domains, eps_dom, omega, ri, src,
                precision):
        eps = complex(float(eps_re), float(eps_im))
        nodes = nodes_nm.detach().cpu().numpy().astype(np.float64)
        prob = Problem.from_arrays(nodes, faces, face_ids, 1e-9, domains)
        solver.set_problem(prob)
        r = list(ri)
        r[eps_dom] = np.sqrt(eps)
        solver.solve_wavelength(omega, r, [src], precision, 1e-12, 30, want_host=False)
        csca, cabs = solver.cross_sections(omega, r[0], [src])
        out = solver.adjoint(omega, r, [src], precision, eps_dom=eps_dom, nodes=True)
        g_nodes = np.zeros((2, len(nodes), 3))
        for d, gd in enumerate(out["dnodes"]):
            np.add.at(g_nodes, (slice(None), prob.node_parent(d)), gd[0] * 1e-9)  # per nm
        ctx.save_for_backward(torch.from_numpy(out["deps"][0].copy()), torch.from_numpy(g_nodes))
        return torch.tensor([csca[0] + cabs[0], cabs[0]], dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad):
        deps, g_nodes = ctx.saved_tensors  # deps [ext, abs][Re, Im]; g_nodes [ext, abs][V][3]
        grad = grad.to(torch.float64)
        d_re = (grad * deps[:, 0]).sum()
        d_im = (grad * deps[:, 1]).sum()
        d_nodes = (grad[:, None, None] * g_nodes).sum(0)
        return d_re, d_im, d_nodes, None, None, None, None, None, None, None, None, None


def cross_sections(solver, eps_re, eps_im, nodes_nm, faces, face_ids, domains, eps_dom, omega, ri, src,
                   precision):
    """[sigma_ext, sigma_abs] (m^2) as a differentiable function of (eps_re, eps_im, nodes_nm)."""
    return CrossSectionsFn.apply(eps_re, eps_im, nodes_nm, solver, faces, face_ids, domains, eps_dom, omega, ri,
                                 src, precision)
