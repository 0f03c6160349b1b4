"""Batched Gaussian FIR: many 2D sfloat images of uneven sizes, each with its own per-axis
sigmas, derivative orders and boundary conditions, in one persistent launch (libdipcu.so's
dipcu_batch_plan_*).  Parameters per image follow PyDIP: per-axis lists in DIPlib order (x
first), a scalar broadcasts to both axes.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import torch

from . import _abi
from .filtering import BoundaryConditionFromString, ParameterError, _array_use_parameter, check, image_desc

__all__ = ["BatchPlan", "device_status", "GRAPH", "AUTOTUNE", "INJECT_INVALID_IMAGE", "INJECT_INVALID_TILE",
           "INJECT_STALLED_COPY"]

GRAPH = 1
AUTOTUNE = 2
INJECT_INVALID_IMAGE = 256
INJECT_INVALID_TILE = 512
INJECT_STALLED_COPY = 1024


def device_status(clear: bool = True) -> int:
    """The device status word (0, or the dipcu_status a kernel reported); synchronises."""
    v = ctypes.c_int(0)
    check(_abi.lib().dipcu_device_status(ctypes.byref(v), int(clear)))
    return v.value


class BatchPlan:
    """A plan over `ins` (2D float32 CUDA tensors) writing `outs` (same shapes, float32).

    ``sigmas``/``orders``/``boundaries`` hold one entry per image (a scalar or a 2-list, x first).
    ``run(stream=None)`` filters every image; with ``graph=True`` that is one CUDA graph launch.
    """

    def __init__(self, ins: Sequence[torch.Tensor], outs: Sequence[torch.Tensor], sigmas, orders, boundaries,
                 truncation: float = 3.0, graph: bool = True, autotune: bool = True, flags: int = 0):
        if len(ins) != len(outs) or len(ins) == 0:
            raise ParameterError("ins and outs must be non-empty lists of the same length")
        n = len(ins)
        descs_in = (_abi.ImageDesc * n)(*[image_desc(t) for t in ins])
        descs_out = (_abi.ImageDesc * n)(*[image_desc(t) for t in outs])
        sig, ords, bcs = [], [], []
        for i in range(n):
            sig += [float(s) for s in _array_use_parameter(sigmas[i], 2, 1.0)]
            ords += [int(o) for o in _array_use_parameter(orders[i], 2, 0)]
            bcs += [BoundaryConditionFromString(b) for b in _array_use_parameter(boundaries[i], 2, "")]
        self._keep = (list(ins), list(outs))
        f = flags | (GRAPH if graph else 0) | (AUTOTUNE if autotune else 0)
        self._plan = ctypes.c_void_p()
        with torch.cuda.device(ins[0].device):
            torch.cuda.synchronize()
            check(_abi.lib().dipcu_batch_plan_create(descs_in, descs_out, n, (ctypes.c_double * (2 * n))(*sig),
                                                     (ctypes.c_uint32 * (2 * n))(*ords),
                                                     (ctypes.c_int32 * (2 * n))(*bcs), float(truncation), f,
                                                     ctypes.byref(self._plan)))
        self.count = n

    def run(self, stream: torch.cuda.Stream | None = None) -> None:
        s = (stream or torch.cuda.current_stream()).cuda_stream
        check(_abi.lib().dipcu_batch_plan_run(self._plan, ctypes.c_void_p(s)))

    def info(self) -> dict:
        ni, tx, ty, g = (ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int())
        check(_abi.lib().dipcu_batch_plan_info(self._plan, ctypes.byref(ni), ctypes.byref(tx), ctypes.byref(ty),
                                               ctypes.byref(g)))
        nk, ng = ctypes.c_int(), ctypes.c_int()
        check(_abi.lib().dipcu_batch_plan_launches(self._plan, ctypes.byref(nk), ctypes.byref(ng)))
        return {"items": ni.value, "tile": (tx.value, ty.value), "grid": g.value, "kernels_per_run": nk.value,
                "grouped_items": ng.value}

    def sigma_table(self) -> torch.Tensor:
        """The plan's device sigma table (2 * count float64, x then y per image), as a tensor view
        over the plan's memory; rewrite it between runs as long as no kernel length changes."""
        ptr = _abi.lib().dipcu_batch_plan_sigmas(self._plan)
        return _device_view(ptr, 2 * self.count, torch.float64, self._keep[0][0].device)

    def close(self) -> None:
        if self._plan:
            _abi.lib().dipcu_batch_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _device_view(ptr: int, n: int, dtype: torch.dtype, device) -> torch.Tensor:
    """A tensor aliasing `n` elements of device memory at `ptr` (owned elsewhere)."""

    class _Iface:
        pass

    iface = _Iface()
    iface.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8" if dtype == torch.float64 else "<f4",
                                      "data": (ptr, False), "version": 3, "strides": None}
    return torch.as_tensor(iface, device=device)
