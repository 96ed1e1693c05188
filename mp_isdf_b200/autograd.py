"""torch.autograd.Function for the nuclear gradient of the ISDF density
functional E = sum_g w_g rho_ISDF(g)^2 (grid points, anchors and weights held
fixed).  Forward runs the B200 adjoint through the C-ABI
(`isdf_energy_gradient`); when the coordinates do not require a gradient it
asks for the energy alone, which skips the gradient sweep.  There is no CPU
path.
"""
from __future__ import annotations

import numpy as np
import torch

from . import capi


class IsdfEnergy(torch.autograd.Function):
    """E(R) for atom coordinates R (natm x 3, bohr, float64 tensor)."""

    @staticmethod
    def forward(ctx_, coords, context, xyz, w, anchors, dm):
        context.set_coords(coords.detach().cpu().numpy())
        if ctx_.needs_input_grad[0]:
            e, g = context.energy_gradient(xyz, w, anchors, dm)
            ctx_.save_for_backward(torch.as_tensor(g, dtype=coords.dtype, device=coords.device))
        else:
            e = context.energy(xyz, w, anchors, dm)
        return torch.tensor(e, dtype=coords.dtype, device=coords.device)

    @staticmethod
    def backward(ctx_, grad_out):
        (g,) = ctx_.saved_tensors
        return grad_out * g, None, None, None, None, None


def isdf_energy(coords: torch.Tensor, context: "capi.Context", xyz: torch.Tensor, w: torch.Tensor,
                anchors, dm) -> torch.Tensor:
    """Differentiable ISDF energy; `coords.grad` receives dE/dR after backward()."""
    return IsdfEnergy.apply(coords, context, xyz, w, np.asarray(anchors), np.asarray(dm))
