"""torch.autograd binding of the adjoint gradient (``vie_power_grad``).

``AbsorbedPower.apply(eps, ctx, edge_mask, opts)`` returns the absorbed power
in the edges of ``edge_mask`` for the per-voxel permittivity ``eps`` (complex
tensor of the grid's shape, the convention of ``Context.set_eps``: the
reference's, Im <= 0 for lossy media; pass ``eps_phys.conj()`` for the
physics convention and autograd conjugates the gradient).  The forward pass
uploads ``eps``, solves, and, when ``eps`` requires a gradient, runs the
adjoint solve at once; backward scales the stored gradient.  torch's
convention for a real loss of a complex input (dL/dRe + i dL/dIm) is the one
the library returns.

All arithmetic is on the GPU through the C ABI; torch only carries the
values.
"""
from __future__ import annotations

import numpy as np
import torch

from . import PREC_FP64, Context


class AbsorbedPower(torch.autograd.Function):
    @staticmethod
    def forward(fctx, eps: torch.Tensor, ctx: Context, edge_mask: np.ndarray, opts: dict | None = None):
        opts = dict(opts or {})
        e = eps.detach().resolve_conj().to("cpu", torch.complex128).numpy()
        ctx.set_eps(e)
        want = eps.requires_grad
        p, g, _, _ = ctx.power_grad(edge_mask, grad=want, solver=opts.get("solver", "bicgstab"),
                                    tol=opts.get("tol", 1e-8), precision=opts.get("precision", PREC_FP64))
        if want:
            fctx.save_for_backward(torch.from_numpy(g).to(eps.device))
        return torch.tensor(p, dtype=torch.float64, device=eps.device)

    @staticmethod
    def backward(fctx, grad_out):
        (g,) = fctx.saved_tensors
        return grad_out.to(g.dtype) * g, None, None, None


def absorbed_power(eps, ctx: Context, edge_mask, **opts):
    """Differentiable absorbed power (see AbsorbedPower)."""
    return AbsorbedPower.apply(eps, ctx, edge_mask, opts)
