"""The allocation-free entry point, dipcu_gauss_fir_noalloc.

Some callers cannot have the library request device memory while they run: their GPU memory is
owned by another allocator (a framework's caching allocator, or a pool reserved at start-up), or
they run long pipelines that must not fail for lack of memory once started.  For them the
filter keeps its pass intermediates in a fixed static device array.  These tests call that entry
point through the C-ABI and check it against the allocating entry point, dipcu_gauss_fir, on
two calls in a row (the array keeps the previous call's contents), and that images larger than
the array are refused.  The file sorts last so that a run stopping at its first failure has run
every other test before it."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _call(fn_name, x, out, sig, ords, bcs):
    import diplib_b200 as dipcu
    from diplib_b200 import _abi
    nd = x.dim()
    din, dout = dipcu.image_desc(x), dipcu.image_desc(out)
    fn = getattr(_abi.lib(), fn_name)
    return fn(ctypes.byref(din), ctypes.byref(dout), (ctypes.c_double * nd)(*sig), (ctypes.c_uint32 * nd)(*ords),
              (ctypes.c_int32 * nd)(*[dipcu.BoundaryConditionFromString(b) for b in bcs]), 3.0,
              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("shape,dtype,sig,ords,bcs", [
    ((96, 130), torch.float32, [2.0, 3.0], [1, 0], ["mirror", "periodic"]),
    ((20, 40, 52), torch.uint16, [1.5, 1.5, 3.0], [0, 2, 1], ["add zeros", "mirror", "third order"]),
    ((17, 33, 29), torch.float64, [1.0, 2.0, 1.5], [0, 1, 0], ["asym mirror", "zero order", "mirror"]),
])
def test_noalloc_matches_allocating_entry_point_twice(shape, dtype, sig, ords, bcs):
    from diplib_b200 import _abi
    assert torch.cuda.is_available()
    dev = torch.device("cuda:0")
    g = torch.Generator(device="cpu").manual_seed(11)
    for call in range(2):                      # second call: new data over the previous contents
        if dtype == torch.uint16:
            x = torch.randint(0, 4096, shape, generator=g, dtype=torch.int32).to(torch.uint16).to(dev)
        else:
            x = torch.rand(shape, generator=g, dtype=dtype).to(dev) * (call + 1)
        odt = torch.float64 if dtype == torch.float64 else torch.float32
        ref = torch.empty(shape, dtype=odt, device=dev)
        got = torch.full(shape, float("nan"), dtype=odt, device=dev)
        assert _call("dipcu_gauss_fir", x, ref, sig, ords, bcs) == 0, _abi.last_error()
        assert _call("dipcu_gauss_fir_noalloc", x, got, sig, ords, bcs) == 0, _abi.last_error()
        torch.cuda.synchronize()
        rng = float(x.double().max() - x.double().min())
        err = float((got.double() - ref.double()).abs().max())
        assert err <= TOL * max(rng, 1.0), (call, err)


def test_noalloc_rejects_images_beyond_the_static_scratch():
    from diplib_b200 import _abi
    dev = torch.device("cuda:0")
    x = torch.zeros((1025, 4096), dtype=torch.float32, device=dev)   # 4 Mi + 4096 samples
    out = torch.empty_like(x)
    st = _call("dipcu_gauss_fir_noalloc", x, out, [1.0, 1.0], [0, 0], ["mirror"])
    assert st == _abi.ERR_INVALID_ARG
    assert "static scratch holds images of at most 4194304 samples" in _abi.last_error()
