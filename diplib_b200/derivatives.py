"""dip::Gradient, dip::GradientMagnitude, dip::Hessian and dip::Laplace (src/linear/derivative.cpp)
with the Gaussian methods, on the B200 Gaussian FIR path: each component is one GaussFIR call
through the C-ABI, written straight into its slice of the output.

Tensor outputs come back planar, the component axis first: ``Gradient`` gives ``(m,) + shape``
for the m axes FindGradientDimensions keeps; ``Hessian`` gives ``(m(m+1)/2,) + shape`` in DIPlib's
symmetric-matrix order (diagonal first, then the elements above it column by column,
include/diplib/library/tensor.h:100-110).  As everywhere in this package the DIPlib axis order
is the reverse of the array's (x is the last array axis) and per-axis parameters are x first.
"""
from __future__ import annotations

import torch

from .filtering import ParameterError, _array_use_parameter, _to_device, _to_host, flex_dtype, Derivative

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


def Gradient(in_, sigmas=(1.0,), method: str = "best", boundaryCondition=(), process=(), truncation: float = 3.0):
    """dip::Gradient (src/linear/derivative.cpp:142-172): the first derivative along every kept
    axis, stacked on a leading component axis."""
    _check_method(method)
    x, was_numpy, dims, sg = _setup(in_, sigmas, process)
    nd = max(1, x.dim())
    out = torch.empty((len(dims),) + tuple(x.shape), dtype=flex_dtype(x.dtype), device=x.device)
    for c, d in enumerate(dims):
        Derivative(x, _order(nd, {d: 1}), sg, method, boundaryCondition, truncation, out=out[c])
    return _to_host(out) if was_numpy else out


def GradientMagnitude(in_, sigmas=(1.0,), method: str = "best", boundaryCondition=(), process=(),
                      truncation: float = 3.0):
    """dip::GradientMagnitude (src/linear/derivative.cpp:174-205): sqrt of the summed squared
    first derivatives (the absolute value for one axis), in the flex type."""
    _check_method(method)
    x, was_numpy, dims, sg = _setup(in_, sigmas, process)
    nd = max(1, x.dim())
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
    for c, (i, j) in enumerate(pairs):
        counts = {dims[i]: 2} if i == j else {dims[i]: 1, dims[j]: 1}
        Derivative(x, _order(nd, counts), sg, method, boundaryCondition, truncation, out=out[c])
    return _to_host(out) if was_numpy else out


def Laplace(in_, sigmas=(1.0,), method: str = "best", boundaryCondition=(), process=(), truncation: float = 3.0):
    """dip::Laplace with the Gaussian methods (src/linear/derivative.cpp:374-418): the sum of the
    second derivatives along the kept axes, accumulated in the flex type."""
    _check_method(method)
    x, was_numpy, dims, sg = _setup(in_, sigmas, process)
    nd = max(1, x.dim())
    out = Derivative(x, _order(nd, {dims[0]: 2}), sg, method, boundaryCondition, truncation)
    if len(dims) > 1:
        tmp = torch.empty_like(out)
        for d in dims[1:]:
            Derivative(x, _order(nd, {d: 2}), sg, method, boundaryCondition, truncation, out=tmp)
            out.add_(tmp)
    return _to_host(out) if was_numpy else out
