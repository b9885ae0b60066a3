"""Differentiable soft-argmin SGM on torch tensors (no reference counterpart).

``soft_sgm(cost, p1, p2, tau)`` returns the expected disparity
dhat = sum_d d * softmax(-S / tau) of the STANDARD 8- (or 4-) path aggregation
S of an (H, W, D) float32/float64 CUDA cost volume.  Forward and backward run
in libtdvb200.so (tdv_soft_sgm_forward / tdv_soft_sgm_backward); this module
only wraps them in a torch.autograd.Function so gradients w.r.t. the cost
volume, P1 and P2 can be checked with torch.autograd.gradcheck.
"""
import ctypes

import torch

from . import _lib as L
from .api import _stream, default_context


def _vol(t):
    if not t.is_cuda or t.dim() != 3 or not t.is_contiguous():
        raise ValueError("cost must be a contiguous (H, W, D) CUDA tensor")
    dt = {torch.float32: L.F32, torch.float64: L.F64}.get(t.dtype)
    if dt is None:
        raise TypeError("cost must be float32 or float64")
    H, W, D = t.shape
    return L.tdv_volume(t.data_ptr(), W, H, D, L.LAYOUT_HWD, dt)


class SoftSGMFunction(torch.autograd.Function):
    @staticmethod
    def forward(fctx, cost, p1, p2, tau, paths, checkpoint, tctx):
        H, W, D = cost.shape
        prm = L.tdv_soft_params(float(p1), float(p2), int(paths), float(tau), int(checkpoint))
        dt = L.F64 if cost.dtype == torch.float64 else L.F32
        nbytes = L.lib().tdv_soft_sgm_tape_bytes(W, H, D, dt, ctypes.byref(prm))
        tape = torch.empty(nbytes, dtype=torch.uint8, device=cost.device)
        dhat = torch.empty((H, W), dtype=cost.dtype, device=cost.device)
        cv = _vol(cost)
        tctx.check(L.lib().tdv_soft_sgm_forward(tctx.handle, ctypes.byref(cv), ctypes.byref(prm),
                                                 ctypes.c_void_p(dhat.data_ptr()),
                                                 ctypes.c_void_p(tape.data_ptr()), nbytes, _stream()))
        fctx.save_for_backward(cost, tape)
        fctx.prm, fctx.tctx, fctx.nbytes = prm, tctx, nbytes
        fctx.pen = (isinstance(p1, torch.Tensor), isinstance(p2, torch.Tensor))
        fctx.pen_dtype = p1.dtype if isinstance(p1, torch.Tensor) else cost.dtype
        return dhat

    @staticmethod
    def backward(fctx, g):
        cost, tape = fctx.saved_tensors
        g = g.contiguous().to(cost.dtype)
        dcost = torch.empty_like(cost)
        dpen = torch.empty(2, dtype=cost.dtype, device=cost.device)
        cv, dv = _vol(cost), _vol(dcost)
        tctx = fctx.tctx
        tctx.check(L.lib().tdv_soft_sgm_backward(tctx.handle, ctypes.byref(cv), ctypes.byref(fctx.prm),
                                                  ctypes.c_void_p(tape.data_ptr()), fctx.nbytes,
                                                  ctypes.c_void_p(g.data_ptr()), ctypes.byref(dv),
                                                  ctypes.c_void_p(dpen.data_ptr()), _stream()))
        d1 = dpen[0].to(fctx.pen_dtype) if fctx.pen[0] else None
        d2 = dpen[1].to(fctx.pen_dtype) if fctx.pen[1] else None
        return dcost, d1, d2, None, None, None, None


def soft_sgm(cost, p1, p2, tau=1.0, paths=8, checkpoint=0, ctx=None):
    """Expected disparity of the soft-argmin SGM; differentiable in cost, p1, p2."""
    tctx = ctx if ctx is not None else default_context(cost.device.index)
    return SoftSGMFunction.apply(cost, p1, p2, tau, paths, checkpoint, tctx)


def soft_sgm_infer(cost, p1, p2, tau=1.0, paths=8, ctx=None):
    """Forward only, no tape (the plain evaluation the adjoint is compared to)."""
    tctx = ctx if ctx is not None else default_context(cost.device.index)
    H, W, D = cost.shape
    prm = L.tdv_soft_params(float(p1), float(p2), int(paths), float(tau), 0)
    dhat = torch.empty((H, W), dtype=cost.dtype, device=cost.device)
    cv = _vol(cost)
    tctx.check(L.lib().tdv_soft_sgm_forward(tctx.handle, ctypes.byref(cv), ctypes.byref(prm),
                                             ctypes.c_void_p(dhat.data_ptr()), None, 0, _stream()))
    return dhat
