"""Differentiable warping, svs/src/warpingOps.py:13-29: an autograd function around
``Warping3D.forward`` / ``Warping3D.backward`` so that a warp inside a training loss back-propagates
into both the image and the flow (the reference's U-Net loop uses it, svs/modules/lit_unet.py:114).

    op = opticalFlow.Warping3D(mesh, INTERPOLATE_CUBIC_HERMITESPLINE, BOUNDARY_MIRROR)
    out = warp(image, flow, op)          # image [Z,Y,X], flow [Z,Y,X,3]; float32 or float64
    out.sum().backward()                 # image.grad, flow.grad
"""
from __future__ import annotations

import torch


class WarpingOpFunction(torch.autograd.Function):
    """forward: op.forward(image, flow); backward: op.backward(image, flow, grad_out) gives the
    gradients with respect to the image (scattered stencil weights) and to the flow (the
    interpolant's spatial derivative at the sample point times grad_out / h)."""

    @staticmethod
    def forward(ctx, image, flow, warpingOp):
        ctx.save_for_backward(image, flow)
        ctx.warpingOp = warpingOp
        return warpingOp.forward(image.contiguous(), flow.contiguous())

    @staticmethod
    def backward(ctx, grad_out):
        image, flow = ctx.saved_tensors
        grad_image, grad_flow = ctx.warpingOp.backward(image.contiguous(), flow.contiguous(),
                                                       grad_out.contiguous())
        return grad_image, grad_flow, None


def warp(image: torch.Tensor, flow: torch.Tensor, warpingOp) -> torch.Tensor:
    return WarpingOpFunction.apply(image, flow, warpingOp)
