"""Differentiable Gaussian FIR for PyTorch (beside PyDIP's dip.Gauss).

``gauss(x, sigma, order, boundary, truncation)`` runs the forward through libdipcu.so and
registers a backward that calls ``dipcu_gauss_fir_backward``: the input gradient is the exact
adjoint of the forward (boundary extension included) and the sigma gradient uses the analytic
derivative of the normalised discrete kernel (its length held fixed).  Parameters follow PyDIP:
per-axis lists in DIPlib order (x first = the last tensor axis); a scalar broadcasts.

``sigma`` may be a Python number/list or a tensor; a tensor that requires grad receives
d(loss)/d(sigma): summed over axes for a scalar sigma, per axis for a vector.  Reading a device
sigma's value costs one device-to-host copy per call.
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi
from .filtering import (BoundaryConditionFromString, GaussFIR, ParameterError, _array_use_parameter, check,
                        flex_dtype, image_desc)

__all__ = ["gauss", "gauss_backward", "structure_tensor", "structure_tensor_backward"]


def _params(nd, sigma, order, boundary):
    if isinstance(sigma, torch.Tensor):
        svals = sigma.detach().reshape(-1).double().cpu().tolist()
    else:
        svals = sigma
    sig = [float(s) for s in _array_use_parameter(svals, nd, 1.0)]
    ords = [int(o) for o in _array_use_parameter(order, nd, 0)]
    bcs = [BoundaryConditionFromString(b) for b in _array_use_parameter(boundary, nd, "")]
    return sig, ords, bcs


def gauss_backward(grad_out: torch.Tensor, x: torch.Tensor | None, sigma, order=0, boundary=(),
                   truncation: float = 3.0, need_input_grad: bool = True, need_sigma_grad: bool = True):
    """(dL/dx or None, dL/dsigma per axis (float64 tensor) or None) for y = GaussFIR(x, ...)."""
    nd = max(1, grad_out.dim())
    sig, ords, bcs = _params(nd, sigma, order, boundary)
    cdt = flex_dtype(x.dtype) if x is not None else grad_out.dtype
    go = grad_out.to(cdt).contiguous()
    gx = torch.empty(go.shape, dtype=cdt, device=go.device) if need_input_grad else None
    gs = torch.zeros(nd, dtype=torch.float64, device=go.device) if need_sigma_grad else None
    d_go = image_desc(go)
    d_x = image_desc(x) if x is not None else None
    d_gx = image_desc(gx) if gx is not None else None
    with torch.cuda.device(go.device):
        check(_abi.lib().dipcu_gauss_fir_backward(
            ctypes.byref(d_go), ctypes.byref(d_x) if d_x is not None else None,
            ctypes.byref(d_gx) if d_gx is not None else None,
            ctypes.c_void_p(gs.data_ptr() if gs is not None else 0),
            (ctypes.c_double * nd)(*sig), (ctypes.c_uint32 * nd)(*ords), (ctypes.c_int32 * nd)(*bcs),
            float(truncation), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return gx, gs


class _GaussFIRFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, sigma_t, sigma, order, boundary, truncation):
        ctx.save_for_backward(x)
        ctx.params = (sigma, order, boundary, truncation)
        ctx.sigma_shape = None if sigma_t is None else sigma_t.shape
        return GaussFIR(x, sigma, order, boundary, truncation)

    @staticmethod
    def backward(ctx, grad_out):
        (x,) = ctx.saved_tensors
        sigma, order, boundary, truncation = ctx.params
        need_x = ctx.needs_input_grad[0]
        need_s = ctx.needs_input_grad[1]
        gx, gs = gauss_backward(grad_out, x, sigma, order, boundary, truncation, need_x, need_s)
        gsig = None
        if need_s:
            if ctx.sigma_shape is not None and len(ctx.sigma_shape) > 0 and int(torch.Size(ctx.sigma_shape).numel()) > 1:
                gsig = gs.to(torch.float32).reshape(ctx.sigma_shape)
            else:
                gsig = gs.sum().reshape(ctx.sigma_shape if ctx.sigma_shape is not None else ())
        if gx is not None and gx.dtype != x.dtype and x.dtype.is_floating_point:
            gx = gx.to(x.dtype)
        return gx, gsig, None, None, None, None


def gauss(x: torch.Tensor, sigma=1.0, order=0, boundary=(), truncation: float = 3.0) -> torch.Tensor:
    """Differentiable dip::GaussFIR of a CUDA tensor (see the module docstring)."""
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise ParameterError("gauss() takes a CUDA tensor")
    sigma_t = sigma if isinstance(sigma, torch.Tensor) else None
    nd = max(1, x.dim())
    sig, _, _ = _params(nd, sigma, order, boundary)
    return _GaussFIRFunction.apply(x, sigma_t, sig, order, boundary, truncation)


def structure_tensor_backward(grad_out: torch.Tensor, x: torch.Tensor, gradient_sigma=1.0, tensor_sigma=5.0,
                              boundary=(), truncation: float = 3.0) -> torch.Tensor:
    """dL/dx for T = StructureTensor(x) given dL/dT (planar, as ``structure_tensor`` returns it).
    The gradient images are recomputed from ``x``."""
    from .analysis import structure_tensor_params
    nd = max(1, x.dim())
    gs, ts, bcs = structure_tensor_params(nd, gradient_sigma, tensor_sigma, "gaussFIR", boundary)
    cdt = flex_dtype(x.dtype)
    go = grad_out.to(cdt)
    gx = torch.empty(x.shape, dtype=cdt, device=x.device)
    d_go, d_x, d_gx = image_desc(go), image_desc(x), image_desc(gx)
    with torch.cuda.device(x.device):
        check(_abi.lib().dipcu_structure_tensor_backward(
            ctypes.byref(d_go), ctypes.byref(d_x), ctypes.byref(d_gx), (ctypes.c_double * nd)(*gs),
            (ctypes.c_double * nd)(*ts), (ctypes.c_int32 * nd)(*bcs), float(truncation),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return gx


class _StructureTensorFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, gradient_sigma, tensor_sigma, boundary, truncation):
        from .analysis import StructureTensor
        ctx.save_for_backward(x)
        ctx.params = (gradient_sigma, tensor_sigma, boundary, truncation)
        return StructureTensor(x, None, gradient_sigma, tensor_sigma, "gaussFIR", boundary, truncation)

    @staticmethod
    def backward(ctx, grad_out):
        (x,) = ctx.saved_tensors
        gx = structure_tensor_backward(grad_out, x, *ctx.params)
        if gx.dtype != x.dtype and x.dtype.is_floating_point:
            gx = gx.to(x.dtype)
        return gx, None, None, None, None


def structure_tensor(x: torch.Tensor, gradient_sigma=1.0, tensor_sigma=5.0, boundary=(),
                     truncation: float = 3.0) -> torch.Tensor:
    """Differentiable dip::StructureTensor (Gaussian FIR, no mask) of a CUDA tensor: shape
    ``(m(m+1)/2,) + x.shape``.  Only ``x`` is saved; the backward recomputes the gradient images."""
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise ParameterError("structure_tensor() takes a CUDA tensor")
    return _StructureTensorFunction.apply(x, gradient_sigma, tensor_sigma, boundary, truncation)
