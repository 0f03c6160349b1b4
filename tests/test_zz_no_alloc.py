"""The allocation-free entry point, dipcu_gauss_fir_noalloc.

Some callers cannot have the library request device memory while they run: their GPU memory is
owned by another allocator (a framework's caching allocator, or a pool reserved at start-up), or
they run long pipelines that must not fail for lack of memory once started.  For them the
filter keeps its pass intermediates in a fixed static device array.  These tests call that entry
point through the C-ABI and check it against the allocating entry point, dipcu_gauss_fir, on
two calls in a row (the array keeps the previous call's contents), and against the oracle; that
it draws nothing from the stream-ordered memory pool (whose high-water mark the allocating entry
point does raise); and that images larger than the array are refused.  The file sorts last so
that a run stopping at its first failure has run every other test before it."""
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


def _pool_high_water_reset():
    """Resets the high-water mark of the device's default stream-ordered memory pool (the pool
    dipcu_gauss_fir's cudaMallocAsync draws from) and returns a reader of it."""
    from cuda.bindings import driver as drv
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(0)
    assert err == rt.cudaError_t.cudaSuccess
    attr = rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh
    (err,) = rt.cudaMemPoolSetAttribute(pool, attr, drv.cuuint64_t(0))
    assert err == rt.cudaError_t.cudaSuccess

    def read() -> int:
        e, v = rt.cudaMemPoolGetAttribute(pool, attr)
        assert e == rt.cudaError_t.cudaSuccess
        return int(v)
    return read


CASES = [
    ((96, 130), torch.float32, torch.float32, [2.0, 3.0], [1, 0], ["mirror", "periodic"]),
    ((20, 40, 52), torch.uint16, torch.float32, [1.5, 1.5, 3.0], [0, 2, 1], ["add zeros", "mirror", "third order"]),
    ((17, 33, 29), torch.float64, torch.float64, [1.0, 2.0, 1.5], [0, 1, 0], ["asym mirror", "zero order", "mirror"]),
    # output type other than the computation type, three passes: both halves of the array in use
    ((18, 35, 41), torch.float32, torch.float64, [1.2, 2.5, 1.0], [1, 0, 2], ["mirror", "first order", "periodic"]),
    ((16, 30, 44), torch.uint16, torch.uint16, [2.0, 1.0, 1.5], [0, 0, 0], ["second order", "mirror", "add zeros"]),
]


def _input(shape, dtype, g, call, dev):
    if dtype == torch.uint16:
        return torch.randint(0, 4096, shape, generator=g, dtype=torch.int32).to(torch.uint16).to(dev)
    return torch.rand(shape, generator=g, dtype=dtype).to(dev) * (call + 1)


@pytest.mark.parametrize("shape,dtype,odt,sig,ords,bcs", CASES)
def test_noalloc_matches_allocating_entry_point_twice(shape, dtype, odt, sig, ords, bcs):
    from diplib_b200 import _abi
    assert torch.cuda.is_available()
    dev = torch.device("cuda:0")
    g = torch.Generator(device="cpu").manual_seed(11)
    for call in range(2):                      # second call: new data over the previous contents
        x = _input(shape, dtype, g, call, dev)
        ref = torch.empty(shape, dtype=odt, device=dev)
        got = torch.full(shape, float("nan"), dtype=odt, device=dev) if odt.is_floating_point else \
            torch.zeros(shape, dtype=odt, device=dev)
        assert _call("dipcu_gauss_fir", x, ref, sig, ords, bcs) == 0, _abi.last_error()
        torch.cuda.synchronize()
        high = _pool_high_water_reset()
        assert _call("dipcu_gauss_fir_noalloc", x, got, sig, ords, bcs) == 0, _abi.last_error()
        torch.cuda.synchronize()
        assert high() == 0, "the allocation-free entry point drew on the stream-ordered pool"
        if odt.is_floating_point:
            rng = float(x.double().max() - x.double().min())
            err = float((got.double() - ref.double()).abs().max())
            assert err <= TOL * max(rng, 1.0), (call, err)
        else:                                   # clamp_cast to an integer output: same samples
            assert torch.equal(got, ref), call


def test_noalloc_matches_the_oracle():
    """Against the restated dip::GaussFIR directly (not only through the allocating entry point)."""
    import oracle
    from diplib_b200 import _abi
    dev = torch.device("cuda:0")
    g = torch.Generator(device="cpu").manual_seed(12)
    for shape, dtype, odt, sig, ords, bcs in CASES:
        x = _input(shape, dtype, g, 0, dev)
        got = torch.zeros(shape, dtype=odt, device=dev)
        assert _call("dipcu_gauss_fir_noalloc", x, got, sig, ords, bcs) == 0, _abi.last_error()
        torch.cuda.synchronize()
        xh = x.cpu().numpy()
        ref = oracle.gauss_fir(xh, sig, ords, bcs, 3.0, out_dtype=got.cpu().numpy().dtype)
        if odt.is_floating_point:
            err = float(np.abs(got.cpu().numpy().astype(np.float64) - ref).max())
            assert err <= TOL * max(float(xh.max()) - float(xh.min()), 1.0), (shape, dtype, err)
        else:
            assert int(np.abs(got.cpu().numpy().astype(np.int64) - ref.astype(np.int64)).max()) <= 1, (shape, dtype)


def test_allocating_entry_point_shows_on_the_pool_probe():
    """The pool probe above sees stream-ordered allocations: the allocating entry point's line-pass
    chain (three passes, output type other than the computation type) raises the high-water mark."""
    from diplib_b200 import _abi
    dev = torch.device("cuda:0")
    x = torch.rand((18, 35, 41), dtype=torch.float32, device=dev)
    out = torch.empty((18, 35, 41), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    high = _pool_high_water_reset()
    assert _call("dipcu_gauss_fir", x, out, [1.2, 2.5, 1.0], [1, 0, 2], ["mirror", "first order", "periodic"]) == 0, \
        _abi.last_error()
    torch.cuda.synchronize()
    assert high() > 0


def test_noalloc_rejects_images_beyond_the_static_scratch():
    from diplib_b200 import _abi
    dev = torch.device("cuda:0")
    x = torch.zeros((1025, 4096), dtype=torch.float32, device=dev)   # 4 Mi + 4096 samples
    out = torch.empty_like(x)
    st = _call("dipcu_gauss_fir_noalloc", x, out, [1.0, 1.0], [0, 0], ["mirror"])
    assert st == _abi.ERR_INVALID_ARG
    assert "static scratch holds images of at most 4194304 samples" in _abi.last_error()
