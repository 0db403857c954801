"""torch.autograd.Function over the C ABI: a gradient test harness only.

``WGradient.apply(eps, sigma, grid, shots, d_obs, gctx)`` returns
J = 0.5 * sum over shots of ||d - d_obs||^2 and, through one
``gj_w_gradient_dev`` call in exact-adjoint mode, saves dJ/d(eps_r) and
dJ/d(sigma) for the backward pass.  eps and sigma are (m, n) CUDA tensors
(depth x lateral); d_obs is (nshots, nr, nt).  It exists so autograd-based
finite-difference checks can drive the CUDA library; the library itself has
no torch dependency.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N


def _colmajor(a: torch.Tensor) -> torch.Tensor:
    """(m, n) tensor -> its column-major flat copy (MATLAB order)."""
    return a.detach().t().contiguous().view(-1)


class WGradient(torch.autograd.Function):
    @staticmethod
    def forward(ctx_, eps, sigma, grid, shots, d_obs, gctx):
        if not (eps.is_cuda and sigma.is_cuda and d_obs.is_cuda):
            raise ValueError("eps, sigma and d_obs must be CUDA tensors")
        m, n = eps.shape
        ef, sf = _colmajor(eps), _colmajor(sigma)
        ge, gs = torch.empty_like(ef), torch.empty_like(sf)
        stream = torch.cuda.current_stream(eps.device).cuda_stream
        gctx.w_gradient_dev(grid, ef, sf, shots, d_obs.contiguous(), ge, gs, mode=N.GJ_ADJ_EXACT, stream=stream)
        ctx_.save_for_backward(ge.view(n, m).t(), gs.view(n, m).t())
        prec = N.GJ_F64 if eps.dtype == torch.float64 else N.GJ_F32
        out = gctx.w_forward(grid, eps.detach().cpu().numpy(), sigma.detach().cpu().numpy(), shots, precision=prec)
        do = d_obs.detach().cpu().numpy()
        J = sum(0.5 * float(np.sum((d - do[k].T) ** 2)) for k, d in enumerate(out["d"]))
        return torch.tensor(J, dtype=torch.float64, device=eps.device)

    @staticmethod
    def backward(ctx_, gJ):
        ge, gs = ctx_.saved_tensors
        s = gJ.to(ge.dtype)
        return s * ge, s * gs, None, None, None, None
