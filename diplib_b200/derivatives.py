"""dip::Gradient, dip::GradientMagnitude, dip::Hessian and dip::Laplace (src/linear/derivative.cpp)
with the Gaussian methods, on the B200 Gaussian FIR path: each component is one GaussFIR call
through the C-ABI, written straight into its slice of the output, as the reference computes them.

``USE_MULTI_OUTPUT = True`` routes the cases the multi-output tile kernel takes (2D/3D input
computed in sfloat, index-mapping or "add zeros" boundary conditions, half-widths up to 8, all
components resolving to the FIR method) through ONE launch that reads the input once
(``dipcu_gauss_fir_multi``): every component, or their sum (Laplace) or root of the summed squares
(GradientMagnitude).  It is off by default because on a B200 that kernel is slower than one
launch of the tile kernels per component (4096^2 Gradient: 318 against 87 us; 192^3: 472 against
130 us): its generic per-tile passes cost more instructions than the second read of the input
saves.

Tensor outputs come back planar, the component axis first: ``Gradient`` gives ``(m,) + shape``
for the m axes FindGradientDimensions keeps; ``Hessian`` gives ``(m(m+1)/2,) + shape`` in DIPlib's
symmetric-matrix order (diagonal first, then the elements above it column by column,
include/diplib/library/tensor.h:100-110).  As everywhere in this package the DIPlib axis order
is the reverse of the array's (x is the last array axis) and per-axis parameters are x first.
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi
from .filtering import (BestGaussMethod, BoundaryConditionFromString, ParameterError, _array_use_parameter, _run,
                        _to_device, _to_host, flex_dtype, image_desc, Derivative)

__all__ = ["Gradient", "GradientMagnitude", "Hessian", "Laplace", "find_gradient_dimensions"]


def find_gradient_dimensions(shape, sigmas, process=None) -> tuple[list, list]:
    """FindGradientDimensions (src/linear/derivative.cpp:120-138) for the Gaussian methods: the
    DIPlib axes with ``process`` set, size > 1 and sigma > 0, and the sigmas broadcast to the
    dimensionality."""
    nd = max(1, len(shape))
    sizes = list(reversed(shape)) if len(shape) else [1]
    sg = [float(s) for s in _array_use_parameter(sigmas, nd, 1.0)]
    pr = [bool(p) for p in _array_use_parameter(process if process is not None else (), nd, True)]
    return [d for d in range(nd) if pr[d] and sizes[d] > 1 and sg[d] > 0.0], sg


def _check_method(method: str) -> None:
    if method == "finitediff":
        raise NotImplementedError("method 'finitediff' is outside the B200 Gaussian FIR path")


def _setup(in_, sigmas, process):
    x, was_numpy = _to_device(in_)
    dims, sg = find_gradient_dimensions(tuple(x.shape), sigmas, process)
    if not dims:
        raise ParameterError("Dimensionality not supported")
    return x, was_numpy, dims, sg


def _order(nd: int, counts: dict) -> list:
    o = [0] * nd
    for d, c in counts.items():
        o[d] += c
    return o


# dipcu_gauss_fir_multi modes
_COMPONENTS, _PRODUCTS, _SUM, _MAGNITUDE = 0, 1, 2, 3

USE_MULTI_OUTPUT = False


def _multi(x: torch.Tensor, orders: list, mode: int, sg: list, method: str, boundaryCondition, truncation: float,
           outs: list) -> bool:
    """All components (or their sum / magnitude) from one read of `x` by the multi-output tile
    kernel, when it takes the case; False (nothing written) when the caller must filter per
    component.  Every component must resolve to the FIR method, as dip::Derivative would pick it."""
    if not USE_MULTI_OUTPUT:
        return False
    m = method[5:] if method[:5] == "gauss" else method
    for o in orders:
        if m == "best":
            if BestGaussMethod(sg, o) != "fir":
                return False
        elif m not in ("fir", "FIR"):
            return False
    nd = max(1, x.dim())
    if nd not in (2, 3) or x.dim() != nd:
        return False
    bcs = [BoundaryConditionFromString(b) for b in _array_use_parameter(boundaryCondition, nd, "")]
    din = image_desc(x)
    flat = [int(v) for o in orders for v in o]
    c_ord = (ctypes.c_uint32 * len(flat))(*flat)
    c_sig = (ctypes.c_double * nd)(*sg)
    c_bc = (ctypes.c_int32 * nd)(*bcs)
    lib = _abi.lib()
    if not lib.dipcu_gauss_fir_multi_supported(ctypes.byref(din), c_ord, len(orders), c_sig, c_bc, float(truncation)):
        return False
    douts = (_abi.ImageDesc * len(outs))(*[image_desc(o) for o in outs])
    _run(x, lib.dipcu_gauss_fir_multi, ctypes.byref(din), douts, len(outs), c_ord, len(orders), mode, c_sig, c_bc,
         float(truncation))
    return True


def Gradient(in_, sigmas=(1.0,), method: str = "best", boundaryCondition=(), process=(), truncation: float = 3.0):
    """dip::Gradient (src/linear/derivative.cpp:142-172): the first derivative along every kept
    axis, stacked on a leading component axis."""
    _check_method(method)
    x, was_numpy, dims, sg = _setup(in_, sigmas, process)
    nd = max(1, x.dim())
    out = torch.empty((len(dims),) + tuple(x.shape), dtype=flex_dtype(x.dtype), device=x.device)
    orders = [_order(nd, {d: 1}) for d in dims]
    if not _multi(x, orders, _COMPONENTS, sg, method, boundaryCondition, truncation, list(out)):
        for c, o in enumerate(orders):
            Derivative(x, o, sg, method, boundaryCondition, truncation, out=out[c])
    return _to_host(out) if was_numpy else out


def GradientMagnitude(in_, sigmas=(1.0,), method: str = "best", boundaryCondition=(), process=(),
                      truncation: float = 3.0):
    """dip::GradientMagnitude (src/linear/derivative.cpp:174-205): sqrt of the summed squared
    first derivatives (the absolute value for one axis), in the flex type."""
    _check_method(method)
    x, was_numpy, dims, sg = _setup(in_, sigmas, process)
    nd = max(1, x.dim())
    if len(dims) > 1:
        out = torch.empty(tuple(x.shape), dtype=flex_dtype(x.dtype), device=x.device)
        if _multi(x, [_order(nd, {d: 1}) for d in dims], _MAGNITUDE, sg, method, boundaryCondition, truncation,
                  [out]):
            return _to_host(out) if was_numpy else out
    out = Derivative(x, _order(nd, {dims[0]: 1}), sg, method, boundaryCondition, truncation)
    if len(dims) == 1:
        out.abs_()
    else:
        out.mul_(out)
        tmp = torch.empty_like(out)
        for d in dims[1:]:
            Derivative(x, _order(nd, {d: 1}), sg, method, boundaryCondition, truncation, out=tmp)
            out.addcmul_(tmp, tmp)
        out.sqrt_()
    return _to_host(out) if was_numpy else out


def Hessian(in_, sigmas=(1.0,), method: str = "best", boundaryCondition=(), process=(), truncation: float = 3.0):
    """dip::Hessian (src/linear/derivative.cpp:330-372): d_ii on the diagonal, then the mixed
    d_ij above it column by column, on a leading component axis."""
    _check_method(method)
    x, was_numpy, dims, sg = _setup(in_, sigmas, process)
    nd = max(1, x.dim())
    m = len(dims)
    pairs = [(i, i) for i in range(m)] + [(i, j) for j in range(1, m) for i in range(j)]
    out = torch.empty((len(pairs),) + tuple(x.shape), dtype=flex_dtype(x.dtype), device=x.device)
    orders = [_order(nd, {dims[i]: 2} if i == j else {dims[i]: 1, dims[j]: 1}) for i, j in pairs]
    if not _multi(x, orders, _COMPONENTS, sg, method, boundaryCondition, truncation, list(out)):
        for c, o in enumerate(orders):
            Derivative(x, o, sg, method, boundaryCondition, truncation, out=out[c])
    return _to_host(out) if was_numpy else out


def Laplace(in_, sigmas=(1.0,), method: str = "best", boundaryCondition=(), process=(), truncation: float = 3.0):
    """dip::Laplace with the Gaussian methods (src/linear/derivative.cpp:374-418): the sum of the
    second derivatives along the kept axes, accumulated in the flex type."""
    _check_method(method)
    x, was_numpy, dims, sg = _setup(in_, sigmas, process)
    nd = max(1, x.dim())
    if len(dims) > 1:
        out = torch.empty(tuple(x.shape), dtype=flex_dtype(x.dtype), device=x.device)
        if _multi(x, [_order(nd, {d: 2}) for d in dims], _SUM, sg, method, boundaryCondition, truncation, [out]):
            return _to_host(out) if was_numpy else out
    out = Derivative(x, _order(nd, {dims[0]: 2}), sg, method, boundaryCondition, truncation)
    if len(dims) > 1:
        tmp = torch.empty_like(out)
        for d in dims[1:]:
            Derivative(x, _order(nd, {d: 2}), sg, method, boundaryCondition, truncation, out=tmp)
            out.add_(tmp)
    return _to_host(out) if was_numpy else out
