"""The differentiable entry point: the render loss of a batch of frames as a
``torch.autograd.Function`` over the library's C ABI (tdi_batch_loss, tdi_batch_loss_backward).

``render_loss(batch, x, lam, L)`` returns, per frame, the negated correlation of the normalised
image gradients of the blurred render and the blurred target -- the image term 3DI's shape fit
minimises (funcs.cu:842-897; the fit scales it by tau_img = 25) -- over the fragments the raster
finds at ``x``, held fixed. Its backward pass is the library's hand-written adjoint: the raster
and the FP64 forward are recomputed, the gradient scattered from pixels to the barycentric
corners with atomics and through the basis transpose to the expression coefficients. Tensors
live on the GPU; ``x`` [F][K+6] (epsilon, tau, u), ``lam`` [F][3] and ``L`` [F] are float32,
the loss and the gradients float64 (returned in the inputs' dtype for the inputs).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _check, default_config, load_library


class RenderLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, batch, cfg, x, lam, L):
        ctx.dtypes = (x.dtype, lam.dtype, L.dtype)
        x, lam, L = (t.detach().contiguous().to(torch.float32) for t in (x, lam, L))
        loss = torch.empty(x.shape[0], dtype=torch.float64, device=x.device)
        stream = C.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)
        _check(load_library().tdi_batch_loss(batch.handle, C.byref(cfg), C.c_void_p(x.data_ptr()),
                                             C.c_void_p(lam.data_ptr()), C.c_void_p(L.data_ptr()),
                                             C.c_void_p(loss.data_ptr()), stream))
        ctx.batch, ctx.cfg = batch, cfg
        ctx.save_for_backward(x, lam, L)
        return loss

    @staticmethod
    def backward(ctx, gloss):
        x, lam, L = ctx.saved_tensors
        gx, glam, gL = loss_gradients(ctx.batch, ctx.cfg, x, lam, L, gloss)
        tx, tl, tL = ctx.dtypes
        return None, None, gx.to(tx), glam.to(tl), gL.to(tL)


def loss_gradients(batch, cfg, x, lam, L, gloss):
    """FP64 gradients of sum_f gloss[f] loss[f] with respect to x, lam and L (the adjoint)."""
    x, lam, L = (t.detach().contiguous().to(torch.float32) for t in (x, lam, L))
    gloss = gloss.detach().contiguous().to(torch.float64)
    gx = torch.empty(x.shape, dtype=torch.float64, device=x.device)
    glam = torch.empty(lam.shape, dtype=torch.float64, device=x.device)
    gL = torch.empty(L.shape, dtype=torch.float64, device=x.device)
    stream = C.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)
    _check(load_library().tdi_batch_loss_backward(
        batch.handle, C.byref(cfg), C.c_void_p(x.data_ptr()), C.c_void_p(lam.data_ptr()),
        C.c_void_p(L.data_ptr()), C.c_void_p(gloss.data_ptr()), C.c_void_p(gx.data_ptr()),
        C.c_void_p(glam.data_ptr()), C.c_void_p(gL.data_ptr()), stream))
    return gx, glam, gL


def render_loss(batch, x, lam, L, cfg=None):
    """Per-frame render loss of the batch's frames (set with Batch.set_frames) at states x."""
    return RenderLoss.apply(batch, cfg if cfg is not None else default_config(), x, lam, L)
