"""dip::StructureTensor on the B200 Gaussian FIR path (src/analysis/structure_tensor.cpp:33-59).

The tensor image comes back planar: shape ``(m(m+1)/2,) + in.shape`` for m gradient axes, the
components in DIPlib's symmetric-matrix order (diagonal first, then the upper triangle row by
row; for 3D: xx, yy, zz, xy, xz, yz with x the LAST array axis).  DIPlib itself stores the
components interleaved (tensor stride 1); the C-ABI takes either layout.
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi
from .filtering import (BestGaussMethod, BoundaryConditionFromString, ParameterError, _array_use_parameter,
                        _to_device, _to_host, check, flex_dtype, image_desc)

__all__ = ["StructureTensor", "structure_tensor_params", "gradient_dims"]


def gradient_dims(shape, grad_sigmas) -> list:
    """FindGradientDimensions (src/linear/derivative.cpp:120-138), DIPlib axis order."""
    sizes = list(reversed(shape)) if len(shape) else [1]
    return [d for d in range(len(sizes)) if sizes[d] > 1 and grad_sigmas[d] > 0.0]


def _resolve_fir(method: str, sigmas, order: int) -> None:
    """dip::Gauss's method resolution (src/linear/derivative.cpp:62-86); only FIR runs here."""
    m = method[5:] if method[:5] == "gauss" else method
    if m == "best":
        m = BestGaussMethod(sigmas, [order] * len(sigmas))
    if m in ("FT", "ft", "IIR", "iir"):
        raise NotImplementedError(f"Gauss method {method!r} (resolved to {m!r}) is outside the B200 FIR path")
    if m not in ("FIR", "fir"):
        raise ParameterError("Invalid flag: " + m)


def structure_tensor_params(nd: int, gradientSigmas, tensorSigmas, method: str, boundaryCondition):
    """Broadcast parameters and resolve ``method`` the way Gradient -> Derivative -> Gauss do."""
    gs = [float(s) for s in _array_use_parameter(gradientSigmas, nd, 1.0)]
    ts = [float(s) for s in _array_use_parameter(tensorSigmas, nd, 5.0)]
    bcs = [BoundaryConditionFromString(b) for b in _array_use_parameter(boundaryCondition, nd, "")]
    if method == "finitediff":
        raise NotImplementedError("StructureTensor method 'finitediff' is outside the B200 Gaussian FIR path")
    if method != "best" and method[:5] != "gauss":
        raise ParameterError("Invalid flag: " + method)
    # Gradient -> Derivative maps "gauss" to "best"; the tensor smoothing calls Gauss directly.
    _resolve_fir("best" if method == "gauss" else method, gs, 1)
    _resolve_fir(method, ts, 0)
    return gs, ts, bcs


def _run(x: torch.Tensor, gs, ts, bcs, truncation: float) -> torch.Tensor:
    nd = max(1, x.dim())
    m = len(gradient_dims(tuple(x.shape), gs))
    if m == 0:
        raise ParameterError("Dimensionality not supported")
    out = torch.empty((m * (m + 1) // 2,) + tuple(x.shape), dtype=flex_dtype(x.dtype), device=x.device)
    din = image_desc(x)
    dout = image_desc(out)
    with torch.cuda.device(x.device):
        check(_abi.lib().dipcu_structure_tensor(
            ctypes.byref(din), ctypes.byref(dout), (ctypes.c_double * nd)(*gs), (ctypes.c_double * nd)(*ts),
            (ctypes.c_int32 * nd)(*bcs), float(truncation), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return out


def StructureTensor(in_, mask=None, gradientSigmas=(1.0,), tensorSigmas=(5.0,), method: str = "best",
                    boundaryCondition=(), truncation: float = 3.0):
    """dip::StructureTensor (include/diplib/analysis.h, src/analysis/structure_tensor.cpp:33-59)
    without a mask, Gaussian FIR derivatives.  Returns a tensor (numpy array for numpy input) of
    shape ``(m(m+1)/2,) + in_.shape``."""
    if mask is not None:
        raise NotImplementedError("StructureTensor with a mask (normalized differential convolution) is outside "
                                  "the B200 Gaussian FIR path")
    x, was_numpy = _to_device(in_)
    if x.dim() < 1 or x.dim() > 3:
        raise ParameterError("Dimensionality not supported")
    gs, ts, bcs = structure_tensor_params(x.dim(), gradientSigmas, tensorSigmas, method, boundaryCondition)
    out = _run(x, gs, ts, bcs, truncation)
    return _to_host(out) if was_numpy else out
