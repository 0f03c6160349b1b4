"""Python host layer of the Gaussian FIR path, mirroring PyDIP's filtering bindings
(pydip/src/filtering.cpp:121-136 in DIPlib): ``Gauss``, ``GaussFIR``, ``Derivative``.

Images are CUDA ``torch.Tensor`` objects (filtered in place on the device) or numpy arrays
(copied to the current CUDA device and back).  As in PyDIP (pydip/src/image.cpp:25-33), the
DIPlib axis order is the reverse of the array order: per-axis parameters (sigmas, orders,
boundary conditions) are listed x first, i.e. for the LAST array axis first.

Every filter call goes through libdipcu.so's C-ABI; nothing here computes pixels.
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Sequence

import numpy as np
import torch

from . import _abi

__all__ = ["Error", "ParameterError", "RunTimeError", "Gauss", "GaussFIR", "Derivative", "BestGaussMethod",
           "SeparableConvolution", "Uniform", "OneDimensionalFilter",
           "BoundaryConditionFromString", "image_desc", "flex_dtype"]


class Error(Exception):
    """dip::Error."""


class ParameterError(Error, ValueError):
    """dip::ParameterError."""


class RunTimeError(Error, RuntimeError):
    """dip::RunTimeError."""


_TORCH_CODES = {
    torch.bool: _abi.BIN, torch.uint8: _abi.UINT8, torch.uint16: _abi.UINT16, torch.uint32: _abi.UINT32,
    torch.uint64: _abi.UINT64, torch.int8: _abi.SINT8, torch.int16: _abi.SINT16, torch.int32: _abi.SINT32,
    torch.int64: _abi.SINT64, torch.float32: _abi.SFLOAT, torch.float64: _abi.DFLOAT,
}
_NP_TO_TORCH = {
    np.dtype(np.bool_): torch.bool, np.dtype(np.uint8): torch.uint8, np.dtype(np.uint16): torch.uint16,
    np.dtype(np.uint32): torch.uint32, np.dtype(np.uint64): torch.uint64, np.dtype(np.int8): torch.int8,
    np.dtype(np.int16): torch.int16, np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64,
    np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
}


def flex_dtype(dtype: torch.dtype) -> torch.dtype:
    """dip::DataType::SuggestFlex (src/library/datatype.cpp:109-124) for real types."""
    if dtype in (torch.uint32, torch.int32, torch.uint64, torch.int64, torch.float64):
        return torch.float64
    if dtype.is_complex:
        raise ParameterError("Data type not supported")
    return torch.float32


def image_desc(t: torch.Tensor) -> _abi.ImageDesc:
    """A dipcu_image_desc of a CUDA tensor: DIPlib axis order (reversed), strides in samples."""
    if t.dtype not in _TORCH_CODES:
        raise ParameterError("Data type not supported")
    if t.dim() > _abi.MAX_DIMS:
        raise ParameterError("Dimensionality not supported")
    d = _abi.ImageDesc()
    d.data = t.data_ptr()
    d.dtype = _TORCH_CODES[t.dtype]
    if t.dim() == 0:
        d.ndims = 1
        d.sizes[0] = 1
        d.strides[0] = 1
        return d
    d.ndims = t.dim()
    for i, (s, st) in enumerate(zip(reversed(t.shape), reversed(t.stride()))):
        d.sizes[i] = int(s)
        d.strides[i] = int(st)
    return d


def _array_use_parameter(values, nd: int, default) -> list:
    """dip::ArrayUseParameter: empty -> default for all, 1 value -> broadcast, nd values -> as is."""
    if values is None:
        values = []
    elif isinstance(values, (int, float, np.integer, np.floating, str)):
        values = [values]
    values = list(values)
    if len(values) == 0:
        return [default] * nd
    if len(values) == 1:
        return values * nd
    if len(values) != nd:
        raise ParameterError("Array parameter has the wrong number of elements")
    return values


_BC_CACHE: dict = {}


def BoundaryConditionFromString(bc: str) -> int:
    """dip::StringToBoundaryCondition (include/diplib/boundary.h:87-103)."""
    code = _BC_CACHE.get(bc)
    if code is None:
        code = _abi.lib().dipcu_bc_from_string(bc.encode())
        if code < 0:
            raise ParameterError("Boundary condition not recognized: " + bc)
        _BC_CACHE[bc] = code
    return code


def BestGaussMethod(sigmas: Sequence[float], orders: Sequence[int]) -> str:
    """BestGaussMethod, src/linear/derivative.cpp:35-58."""
    if any(o > 3 for o in orders):
        return "ft"
    if any(0.0 < s < 0.8 for s in sigmas):
        return "ft"
    if any(s > 10 for s in sigmas):
        return "iir"
    return "fir"


_STATUS_ERRORS = {
    _abi.ERR_INVALID_ARG: ParameterError,
    _abi.ERR_UNSUPPORTED_DTYPE: ParameterError,
    _abi.ERR_UNSUPPORTED_BC: ParameterError,
    _abi.ERR_ORDER_GT_3: ParameterError,
    _abi.ERR_SIZES_DONT_MATCH: ParameterError,
    _abi.ERR_KERNEL_TOO_LARGE: ParameterError,
    _abi.ERR_CUDA: RunTimeError,
    _abi.ERR_TIMEOUT: RunTimeError,
}


def check(status: int) -> None:
    if status != _abi.OK:
        raise _STATUS_ERRORS.get(status, RunTimeError)(_abi.last_error())


def _to_device(img):
    """(tensor on the current CUDA device, was_numpy)."""
    if isinstance(img, torch.Tensor):
        if not img.is_cuda:
            raise ParameterError("tensor images must live on a CUDA device")
        return img, False
    arr = np.asarray(img)
    if arr.dtype not in _NP_TO_TORCH:
        raise ParameterError("Data type not supported")
    # torch.from_numpy lacks some unsigned types; go through a byte view.
    t = torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8)).view(_NP_TO_TORCH[arr.dtype]).reshape(arr.shape)
    return t.to("cuda", non_blocking=False), True


def _to_host(t: torch.Tensor) -> np.ndarray:
    np_dt = {v: k for k, v in _NP_TO_TORCH.items()}[t.dtype]
    host = t.contiguous().cpu()
    return host.view(torch.uint8).numpy().view(np_dt).reshape(tuple(host.shape))


def _shares_memory(a: torch.Tensor, b: torch.Tensor) -> bool:
    """True when the two tensors' storages overlap (DIPlib strips such an output first)."""
    sa, sb = a.untyped_storage(), b.untyped_storage()
    a0, b0 = sa.data_ptr(), sb.data_ptr()
    return a0 < b0 + max(1, sb.nbytes()) and b0 < a0 + max(1, sa.nbytes())


def GaussFIR(in_, sigmas: Iterable[float] | float = (1.0,), derivativeOrder: Iterable[int] | int = (0,),
             boundaryCondition: Iterable[str] | str = (), truncation: float = 3.0, *, out=None):
    """dip::GaussFIR (include/diplib/linear.h:300-318, src/linear/gauss.cpp:238-286).

    ``out``: optional CUDA tensor of the input's shape.  Its type is kept (DIPlib's protected
    output: computation in the flex type, clamp_cast on the final write); if it shares memory
    with the input the result goes through a fresh buffer first, as DIPlib strips such outputs.
    Returns the output (a tensor, or a numpy array for numpy input).
    """
    x, was_numpy = _to_device(in_)
    nd = max(1, x.dim())
    sig = [float(s) for s in _array_use_parameter(sigmas, nd, 1.0)]
    ords = [int(o) for o in _array_use_parameter(derivativeOrder, nd, 0)]
    bcs = [BoundaryConditionFromString(b) for b in _array_use_parameter(boundaryCondition, nd, "")]
    if any(o < 0 for o in ords):
        raise ParameterError("derivative orders must be non-negative")
    if out is None:
        res = torch.empty(x.shape, dtype=flex_dtype(x.dtype), device=x.device)
        target = None
    else:
        if not isinstance(out, torch.Tensor) or out.device != x.device:
            raise ParameterError("out must be a tensor on the input's device")
        if tuple(out.shape) != tuple(x.shape):
            raise ParameterError("Sizes don't match")
        if _shares_memory(out, x):
            res = torch.empty(out.shape, dtype=out.dtype, device=out.device)
            target = out
        else:
            res = out
            target = None
    din = image_desc(x)
    dout = image_desc(res)
    args = (ctypes.byref(din), ctypes.byref(dout), (ctypes.c_double * nd)(*sig), (ctypes.c_uint32 * nd)(*ords),
            (ctypes.c_int32 * nd)(*bcs), float(truncation))
    if x.device.index == torch.cuda.current_device():
        check(_abi.lib().dipcu_gauss_fir(*args, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    else:
        with torch.cuda.device(x.device):
            check(_abi.lib().dipcu_gauss_fir(*args, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    if target is not None:
        target.copy_(res)
        res = target
    return _to_host(res) if was_numpy else res


def _as_list(v) -> list:
    return [v] if isinstance(v, str) else list(v)


def _prepare_out(x: torch.Tensor, out):
    """(result tensor, tensor to copy it into afterwards or None) for an optional `out`, with
    DIPlib's rules: the output's type is kept when given (protected output), and an output sharing
    memory with the input gets a fresh buffer first."""
    if out is None:
        return torch.empty(x.shape, dtype=flex_dtype(x.dtype), device=x.device), None
    if not isinstance(out, torch.Tensor) or out.device != x.device:
        raise ParameterError("out must be a tensor on the input's device")
    if tuple(out.shape) != tuple(x.shape):
        raise ParameterError("Sizes don't match")
    if _shares_memory(out, x):
        return torch.empty(out.shape, dtype=out.dtype, device=out.device), out
    return out, None


def _run(x: torch.Tensor, fn, *args) -> None:
    if x.device.index == torch.cuda.current_device():
        check(fn(*args, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    else:
        with torch.cuda.device(x.device):
            check(fn(*args, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))


class OneDimensionalFilter:
    """dip::OneDimensionalFilter (include/diplib/linear.h:84-92): real `filter` weights, `origin`
    (-1: the centre) and `symmetry` ("general", "even", "odd", "conj", "d-even", "d-odd", "d-conj")."""

    def __init__(self, filter=(), origin: int = -1, symmetry: str = "general", isComplex: bool = False):
        self.filter = [float(v) for v in filter]
        self.origin = int(origin)
        self.symmetry = symmetry
        self.isComplex = bool(isComplex)


def SeparableConvolution(in_, filter, boundaryCondition=(), process=(), *, out=None):
    """dip::SeparableConvolution (include/diplib/linear.h:114-129, src/linear/convolution.cpp:319-421)
    for real filters: `filter` is one OneDimensionalFilter (or a dict with the same keys) used along
    every axis, or one per axis (DIPlib order, x first); `process` (optional) one flag per axis."""
    x, was_numpy = _to_device(in_)
    nd = max(1, x.dim())
    filters = filter if isinstance(filter, (list, tuple)) else [filter]
    filters = [OneDimensionalFilter(**f) if isinstance(f, dict) else f for f in filters]
    if len(filters) not in (1, nd):
        raise ParameterError("Array parameter has the wrong number of elements")
    if any(f.isComplex for f in filters):
        raise NotImplementedError("complex filters are outside the B200 real-valued path")
    syms = []
    for f in filters:
        if f.symmetry not in _abi.SYMMETRY:
            raise ParameterError("Symmetry string not recognized: " + f.symmetry)
        syms.append(_abi.SYMMETRY[f.symmetry])
    bcs = [BoundaryConditionFromString(b) for b in _array_use_parameter(boundaryCondition, nd, "")]
    proc = list(process) if process else []
    if proc and len(proc) != nd:
        raise ParameterError("Array parameter has the wrong number of elements")
    weights = [(ctypes.c_double * max(1, len(f.filter)))(*f.filter) for f in filters]
    descs = (_abi.Filter1D * len(filters))(*[
        _abi.Filter1D(ctypes.cast(w, ctypes.POINTER(ctypes.c_double)), len(f.filter), f.origin, sy)
        for w, f, sy in zip(weights, filters, syms)])
    res, target = _prepare_out(x, out)
    din, dout = image_desc(x), image_desc(res)
    pr = (ctypes.c_uint8 * nd)(*[1 if p_ else 0 for p_ in proc]) if proc else None
    _run(x, _abi.lib().dipcu_separable_convolution, ctypes.byref(din), ctypes.byref(dout), descs, len(filters),
         (ctypes.c_int32 * nd)(*bcs), pr)
    if target is not None:
        target.copy_(res)
        res = target
    return _to_host(res) if was_numpy else res


def Uniform(in_, kernel=7, boundaryCondition=(), *, shape: str = "rectangular", out=None):
    """dip::Uniform (include/diplib/linear.h:262-275, src/linear/uniform.cpp:147-163) with a
    rectangular kernel: `kernel` holds the per-axis sizes (a scalar broadcasts; DIPlib order).  Other
    kernel shapes (the pixel-table path) are outside this implementation."""
    if shape != "rectangular":
        raise NotImplementedError("only rectangular uniform kernels are implemented on the B200 path")
    x, was_numpy = _to_device(in_)
    nd = max(1, x.dim())
    sizes = [float(v) for v in _array_use_parameter(kernel, nd, 7.0)]
    bcs = [BoundaryConditionFromString(b) for b in _array_use_parameter(boundaryCondition, nd, "")]
    res, target = _prepare_out(x, out)
    din, dout = image_desc(x), image_desc(res)
    _run(x, _abi.lib().dipcu_uniform, ctypes.byref(din), ctypes.byref(dout), (ctypes.c_double * nd)(*sizes),
         (ctypes.c_int32 * nd)(*bcs))
    if target is not None:
        target.copy_(res)
        res = target
    return _to_host(res) if was_numpy else res


def GaussFT(in_, sigmas: Iterable[float] | float = (1.0,), derivativeOrder: Iterable[int] | int = (0,),
            truncation: float = 3.0, inRepresentation: str = "spatial", outRepresentation: str = "spatial",
            boundaryCondition: Iterable[str] | str = (), *, out=None):
    """dip::GaussFT (include/diplib/linear.h:365-390, src/linear/gauss.cpp:397-487) with spatial
    input and output.  ``boundaryCondition`` empty: the transform covers exactly the image; else
    the image is first extended by it (one value for all axes, or one per axis).  ``out`` as in
    GaussFIR."""
    for rep in (inRepresentation, outRepresentation):
        if rep not in ("spatial", "frequency"):
            raise ParameterError("Invalid flag: " + rep)
    if inRepresentation != "spatial" or outRepresentation != "spatial":
        raise NotImplementedError("GaussFT on the B200 path takes and returns spatial images")
    x, was_numpy = _to_device(in_)
    if x.dtype.is_complex:
        raise NotImplementedError("complex images are outside the B200 real-valued path")
    nd = max(1, x.dim())
    sig = [float(s) for s in _array_use_parameter(sigmas, nd, 1.0)]
    ords = [int(o) for o in _array_use_parameter(derivativeOrder, nd, 0)]
    if any(o < 0 for o in ords):
        raise ParameterError("derivative orders must be non-negative")
    bcl = list(boundaryCondition) if not isinstance(boundaryCondition, str) else [boundaryCondition]
    bcs = [BoundaryConditionFromString(b) for b in _array_use_parameter(bcl, nd, "")] if bcl else []
    res, target = _prepare_out(x, out)
    din, dout = image_desc(x), image_desc(res)
    _run(x, _abi.lib().dipcu_gauss_ft, ctypes.byref(din), ctypes.byref(dout), (ctypes.c_double * nd)(*sig),
         (ctypes.c_uint32 * nd)(*ords), float(truncation), (ctypes.c_int32 * max(1, len(bcs)))(*bcs), len(bcs))
    if target is not None:
        target.copy_(res)
        res = target
    return _to_host(res) if was_numpy else res


def GaussIIR(in_, sigmas: Iterable[float] | float = (1.0,), derivativeOrder: Iterable[int] | int = (0,),
             boundaryCondition: Iterable[str] | str = (), filterOrder: Iterable[int] | int = (),
             designMethod: str = "discrete time fit", truncation: float = 3.0, *, out=None):
    """dip::GaussIIR (include/diplib/linear.h:407-428, src/linear/gaussiir.cpp:725-790; PyDIP
    pydip/src/filtering.cpp:129-132): the recursive Gaussian of van Vliet, Young and Verbeek,
    derivative orders 0-4, computed in dfloat on the device.  ``filterOrder`` empty: order + 3 (5
    above order 2) per axis; ``designMethod``: "discrete time fit" or "forward backward"."""
    x, was_numpy = _to_device(in_)
    nd = max(1, x.dim())
    sig = [float(s) for s in _array_use_parameter(sigmas, nd, 1.0)]
    ords = [int(o) for o in _array_use_parameter(derivativeOrder, nd, 0)]
    bcs = [BoundaryConditionFromString(b) for b in _array_use_parameter(boundaryCondition, nd, "")]
    fo = _as_list(filterOrder) if not isinstance(filterOrder, int) else [filterOrder]
    fo = [int(v) for v in _array_use_parameter(fo, nd, 3)] if fo else None
    if any(o < 0 for o in ords):
        raise ParameterError("derivative orders must be non-negative")
    if designMethod == "forward backward":
        design = _abi.IIR_FORWARD_BACKWARD
    elif designMethod == "discrete time fit":
        design = _abi.IIR_DISCRETE_TIME_FIT
    else:
        raise ParameterError("Invalid flag: " + designMethod)
    res, target = _prepare_out(x, out)
    din, dout = image_desc(x), image_desc(res)
    _run(x, _abi.lib().dipcu_gauss_iir, ctypes.byref(din), ctypes.byref(dout), (ctypes.c_double * nd)(*sig),
         (ctypes.c_uint32 * nd)(*ords), (ctypes.c_int32 * nd)(*bcs), (ctypes.c_uint32 * nd)(*fo) if fo else None,
         design, float(truncation))
    if target is not None:
        target.copy_(res)
        res = target
    return _to_host(res) if was_numpy else res


def Gauss(in_, sigmas=(1.0,), derivativeOrder=(0,), method: str = "best", boundaryCondition=(),
          truncation: float = 3.0, *, out=None):
    """dip::Gauss (src/linear/derivative.cpp:62-86): the "gauss" prefix is stripped and "best"
    resolved by BestGaussMethod; the FIR, FT and IIR methods (IIR with the reference's defaults:
    recursion order per derivative order, "discrete time fit")."""
    m = method[5:] if method[:5] == "gauss" else method
    x_nd = max(1, (in_.dim() if isinstance(in_, torch.Tensor) else np.asarray(in_).ndim))
    if m == "best":
        m = BestGaussMethod(_array_use_parameter(sigmas, x_nd, 1.0), _array_use_parameter(derivativeOrder, x_nd, 0))
    if m in ("FIR", "fir"):
        return GaussFIR(in_, sigmas, derivativeOrder, boundaryCondition, truncation, out=out)
    if m in ("FT", "ft"):
        # For GaussFT the empty boundary condition is not dip::Gauss's default (derivative.cpp:76-79).
        bc = boundaryCondition if len(_as_list(boundaryCondition)) else ["default"]
        return GaussFT(in_, sigmas, derivativeOrder, truncation, "spatial", "spatial", bc, out=out)
    if m in ("IIR", "iir"):
        return GaussIIR(in_, sigmas, derivativeOrder, boundaryCondition, (), "discrete time fit", truncation, out=out)
    raise ParameterError("Invalid flag: " + m)


def Derivative(in_, derivativeOrder=(0,), sigmas=(1.0,), method: str = "best", boundaryCondition=(),
               truncation: float = 3.0, *, out=None):
    """dip::Derivative (src/linear/derivative.cpp:88-116), Gaussian methods."""
    if method == "best" or method[:5] == "gauss":
        return Gauss(in_, sigmas, derivativeOrder, "best" if method == "gauss" else method, boundaryCondition,
                     truncation, out=out)
    raise ParameterError("Invalid flag: " + method)
