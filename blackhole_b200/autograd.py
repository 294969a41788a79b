"""torch.autograd wrapper of the discrete adjoint (for checking and for use in
torch optimisation loops).

``luminance_loss(params, target, cfg, renderer)`` returns the loss
sum((Y - target)^2) of the binary64 frame of ``cfg`` with (spin, inclination,
eddington, disc_r_out) taken from the 4-element tensor ``params``; its
backward is the gradient bh_gpu_adjoint computes, scaled by the incoming
gradient.  The render and the adjoint run in one call during forward.
"""
from __future__ import annotations

import copy

import numpy as np


def _torch():
    import torch

    return torch


class _LuminanceLoss:
    fn = None

    @classmethod
    def get(cls):
        if cls.fn is None:
            torch = _torch()

            class Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, params, target, cfg, renderer):
                    p = params.detach().to("cpu", torch.float64).numpy()
                    c = copy.deepcopy(cfg)
                    c.spin, c.cam.theta, c.eddington, c.disc_r_out = (float(x) for x in p)
                    t = target.detach().to("cpu", torch.float32).numpy() if hasattr(target, "detach") \
                        else np.asarray(target, dtype=np.float32)
                    g = renderer.adjoint(c, t)
                    grad = torch.tensor([g["d_spin"], g["d_inclination"], g["d_eddington"], g["d_r_out"]],
                                        dtype=params.dtype, device=params.device)
                    ctx.save_for_backward(grad)
                    return torch.tensor(g["loss"], dtype=params.dtype, device=params.device)

                @staticmethod
                def backward(ctx, grad_out):
                    (grad,) = ctx.saved_tensors
                    return grad_out * grad, None, None, None

            cls.fn = Fn
        return cls.fn


def luminance_loss(params, target, cfg, renderer):
    """Loss of the frame at `params` = (spin, inclination, eddington, r_out)."""
    return _LuminanceLoss.get().apply(params, target, cfg, renderer)
