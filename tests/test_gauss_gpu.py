"""Parity of the CUDA Gaussian FIR path (through libdipcu.so's C-ABI) with the oracle.

Bar (the task's parity bar for this path): max |GPU - oracle| <= 1e-5 * (input range) for
float outputs; DIPlib's pass-by-pass float semantics differ from the fused kernels only in
rounding order."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch

import oracle
from tests.golden.make_golden import CASES, make_input

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-5


def dip():
    import diplib_b200
    return diplib_b200


def to_dev(x: np.ndarray) -> torch.Tensor:
    return dip().filtering._to_device(x)[0]


def tol_for(x: np.ndarray) -> float:
    xf = x.astype(np.float64)
    rng = float(xf.max() - xf.min()) if xf.size else 0.0
    return TOL * max(rng, 1.0)


def assert_close(got: np.ndarray, ref: np.ndarray, x: np.ndarray, what=""):
    assert got.shape == ref.shape and got.dtype == ref.dtype, what
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(got)), what
    if ref.dtype.kind == "f":
        err = np.abs(got[fin].astype(np.float64) - ref[fin].astype(np.float64))
        big = np.abs(ref[fin]) > 1e30          # "add max"/"add min" halos: compare relatively
        bound = np.where(big, 1e-5 * np.abs(ref[fin]), tol_for(x))
        assert np.all(err <= bound), f"{what}: max err {err.max() if err.size else 0} > {tol_for(x)}"
    else:
        assert np.abs(got.astype(np.int64) - ref.astype(np.int64)).max() <= 1, what


def test_golden_fixtures(cuda):
    ref = np.load(os.path.join(GOLDEN, "gauss_ref.npz"))
    for name, seed, shape, dtype, sig, ords, bcs, trunc in CASES:
        x = make_input(seed, shape, dtype)
        got = dip().GaussFIR(x, sig, ords, bcs, trunc)
        assert_close(got, ref[name], x, name)


@pytest.mark.parametrize("seed", range(6))
def test_fuzz_against_oracle(cuda, seed):
    rng = np.random.default_rng(1000 + seed)
    bcs = ["mirror", "asym mirror", "antisym reflect", "periodic", "asym periodic", "add zeros", "zero order",
           "first order", "second order", "third order"]
    for it in range(25):
        nd = int(rng.integers(1, 5))
        shape = tuple(int(rng.integers(1, 40 if nd < 3 else 18)) for _ in range(nd))
        dtype = [np.float32, np.uint16, np.uint8, np.int16, np.float64, np.int32, np.bool_][int(rng.integers(0, 7))]
        x = make_input(int(rng.integers(0, 1 << 30)), shape, dtype)
        sig = [float(rng.choice([0.0, 0.6, 1.0, 1.5, 2.5, 4.0])) for _ in range(nd)]
        ords = [int(rng.integers(0, 4)) for _ in range(nd)]
        bc = [str(rng.choice(bcs)) for _ in range(nd)]
        tr = float(rng.choice([2.0, 3.0, 4.5]))
        ref = oracle.gauss_fir(x, sig, ords, bc, tr)
        got = dip().GaussFIR(x, sig, ords, bc, tr)
        assert_close(got, ref, x, f"{it}: {shape} {np.dtype(dtype)} {sig} {ords} {bc} {tr}")


@pytest.mark.parametrize("case", [
    # (shape numpy order, dtype, sigmas x-first, orders, bcs) -- fused-kernel configurations
    ((256, 320), np.float32, [2.0, 2.0], [0, 0], ["mirror"]),
    ((130, 200), np.float32, [3.0, 3.0], [1, 0], ["periodic"]),
    ((130, 200), np.float32, [3.0, 3.0], [0, 1], ["add zeros"]),
    ((99, 77), np.float32, [3.0, 3.0], [2, 0], ["asym mirror", "zero order"]),
    ((70, 90), np.uint16, [2.0, 2.0], [0, 0], ["asym periodic"]),
    ((40, 48, 70), np.uint16, [1.5, 1.5, 3.0], [0, 0, 0], ["mirror"]),
    ((40, 48, 70), np.uint16, [1.5, 1.5, 3.0], [1, 0, 0], ["mirror"]),
    ((33, 21, 50), np.uint16, [1.5, 1.5, 3.0], [0, 0, 0], ["periodic", "add zeros", "zero order"]),
    ((30, 40, 50), np.float32, [1.0, 1.0, 1.0], [1, 0, 0], ["mirror"]),
    ((30, 40, 50), np.float32, [1.0, 1.0, 1.0], [0, 0, 1], ["asym mirror"]),
    ((40, 40, 40), np.float32, [4.0, 4.0, 4.0], [0, 0, 0], ["mirror"]),
    ((6, 50, 70), np.float32, [2.0, 2.0, 0.0], [0, 0, 0], ["mirror"]),   # z unfiltered: batch axis
    ((30, 37, 70), np.uint16, [1.5, 1.5, 3.0], [0, 0, 0], ["asym mirror"]),             # mapped y pass
    ((30, 37, 70), np.float32, [1.5, 1.5, 3.0], [0, 0, 0], ["asym mirror", "add zeros", "mirror"]),  # fix-up, negated
    ((20, 9, 70), np.uint16, [1.5, 1.5, 3.0], [0, 0, 0], ["mirror"]),                   # halo leaves the box
    ((25, 30, 130), np.uint16, [1.5, 1.5, 3.0], [1, 0, 0], ["zero order", "periodic", "asym periodic"]),
    ((300, 16, 64), np.uint16, [1.5, 1.5, 3.0], [0, 0, 0], ["mirror"]),                 # long z, several chunks
])
def test_fused_configs_against_oracle(cuda, case):
    shape, dtype, sig, ords, bcs = case
    x = make_input(77, shape, dtype)
    ref = oracle.gauss_fir(x, sig, ords, bcs, 3.0)
    got = dip().GaussFIR(x, sig, ords, bcs, 3.0)
    assert_close(got, ref, x, str(case))


def test_strided_views(cuda):
    x = make_input(3, (50, 60, 8), np.float32)
    xt = to_dev(x)
    views = [xt[:, :, 3], xt[::2, 1:50:3, 5], xt.permute(2, 0, 1), xt.transpose(0, 1), xt[4:40, :, 1:7]]
    for v in views:
        host = v.cpu().numpy()
        nd = v.dim()
        ref = oracle.gauss_fir(np.ascontiguousarray(host), [1.5, 2.0, 1.0][:nd], [1, 0, 0][:nd], ["mirror"], 3.0)
        got = dip().GaussFIR(v, [1.5, 2.0, 1.0][:nd], [1, 0, 0][:nd], ["mirror"], 3.0).cpu().numpy()
        assert_close(got, ref, host, str(v.shape))


def test_negative_strides_through_c_abi(cuda):
    import ctypes
    from diplib_b200 import _abi
    x = make_input(4, (37, 45), np.float32)
    xt = to_dev(x)
    out = torch.empty_like(xt)
    din = dip().image_desc(xt)
    # View the rows in reverse order: origin at the last row, negative y stride.
    din.data = xt[-1].data_ptr()
    din.strides[1] = -x.shape[1]
    dout = dip().image_desc(out)
    nd = 2
    st = _abi.lib().dipcu_gauss_fir(ctypes.byref(din), ctypes.byref(dout), (ctypes.c_double * nd)(1.2, 2.3),
                                    (ctypes.c_uint32 * nd)(0, 1), (ctypes.c_int32 * nd)(0, 3), 3.0,
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, _abi.last_error()
    ref = oracle.gauss_fir(np.ascontiguousarray(x[::-1]), [1.2, 2.3], [0, 1], ["mirror", "periodic"], 3.0)
    assert_close(out.cpu().numpy(), ref, x, "negative stride")


def test_protected_output_types(cuda):
    x = make_input(5, (30, 40), np.float32) * 300.0
    xt = to_dev(x)
    for tdt, ndt in [(torch.uint8, np.uint8), (torch.int16, np.int16), (torch.float64, np.float64)]:
        out = torch.empty(x.shape, dtype=tdt, device=cuda)
        dip().GaussFIR(xt, [2.0], [0], ["mirror"], 3.0, out=out)
        ref = oracle.gauss_fir(x, [2.0], [0], ["mirror"], 3.0, out_dtype=ndt)
        got = out.cpu().numpy()
        if ndt == np.float64:
            np.testing.assert_allclose(got, ref, atol=tol_for(x))
        else:
            assert np.abs(got.astype(np.int64) - ref.astype(np.int64)).max() <= 1, tdt


def test_in_place_output_is_stripped(cuda):
    x = make_input(6, (40, 50), np.float32)
    xt = to_dev(x)
    ref = oracle.gauss_fir(x, [2.0], [0], ["mirror"], 3.0)
    dip().GaussFIR(xt, [2.0], [0], ["mirror"], 3.0, out=xt)
    assert_close(xt.cpu().numpy(), ref, x, "in place")


def test_errors_mirror_reference(cuda):
    d = dip()
    x = torch.zeros((8, 8), device=cuda)
    with pytest.raises(d.ParameterError, match="Gaussian FIR filter not implemented for order > 3"):
        d.GaussFIR(x, [1.0], [4])
    with pytest.raises(d.ParameterError, match="Boundary condition not recognized: nope"):
        d.GaussFIR(x, [1.0], [0], ["nope"])
    with pytest.raises(d.ParameterError, match="Array parameter has the wrong number of elements"):
        d.GaussFIR(x, [1.0, 2.0, 3.0])
    with pytest.raises(d.ParameterError, match="Sizes don't match"):
        d.GaussFIR(x, [1.0], out=torch.zeros((8, 9), device=cuda))
    with pytest.raises(d.ParameterError, match="Invalid flag"):
        d.Gauss(x, [1.0], [0], "bogus")
    # order > 3 on an unprocessed axis is not an error (gauss.cpp only checks processed axes)
    d.GaussFIR(x, [1.0, 0.0], [0, 5])


def test_gauss_best_method_dispatch(cuda):
    x = make_input(8, (32, 32), np.float32)
    ref = oracle.gauss_fir(x, [2.0], [0], ["mirror"], 3.0)
    assert_close(dip().Gauss(x, 2.0), ref, x, "best")
    assert_close(dip().Gauss(x, [2.0], [0], "gaussFIR"), ref, x, "gaussFIR")
    # sigma < 0.8 resolves to the FT method ("default" boundary condition), sigma > 10 to IIR
    assert_close(dip().Gauss(x, [0.5]), oracle.gauss_ft(x, [0.5], [0], 3.0, ["mirror"]), x, "best -> FT")
    assert_close(dip().Gauss(x, [12.0], [1]), oracle.gauss_iir(x, [12.0], [1], ["mirror"]), x, "best -> IIR")


def test_device_weights_match_oracle(cuda):
    """K0 on the device: every tap equals the reference's MakeHalfGaussian cast to float, bit for bit."""
    from diplib_b200 import _abi
    sig = [0.8, 1.0, 1.5, 2.0, 3.0, 4.0, 8.0, 11.0] + [float(s) for s in
                                                      np.round(np.random.default_rng(5).uniform(0.3, 20.0, 200), 3)]
    pairs = [(s, o) for s in sig for o in range(4)]
    stride = 96
    s_d = torch.tensor([p[0] for p in pairs], dtype=torch.float64, device=cuda)
    o_d = torch.tensor([p[1] for p in pairs], dtype=torch.int32, device=cuda)
    w = torch.zeros((len(pairs), stride), dtype=torch.float32, device=cuda)
    dw = torch.zeros_like(w)
    ln = torch.zeros(len(pairs), dtype=torch.int32, device=cuda)
    st = _abi.lib().dipcu_make_gauss_weights(s_d.data_ptr(), o_d.data_ptr(), len(pairs), 3.0, w.data_ptr(),
                                             dw.data_ptr(), ln.data_ptr(), stride,
                                             torch.cuda.current_stream().cuda_stream)
    assert st == 0
    torch.cuda.synchronize()
    w = w.cpu().numpy()
    ln = ln.cpu().numpy()
    for i, (s, o) in enumerate(pairs):
        ref = oracle.half_gaussian(s, o, 3.0, False)[::-1].astype(np.float32)
        assert ln[i] == ref.size
        np.testing.assert_array_equal(w[i, :ref.size], ref, err_msg=f"sigma {s} order {o}")


def test_launch_counter_counts_kernel_launches(cuda):
    """dipcu_launch_count: one fused-tile launch per plain 2D float GaussFIR call, none for a call
    that filters nothing (every sigma 0: a conversion copy only when the types differ)."""
    import torch
    import diplib_b200 as dip
    from diplib_b200 import _abi
    x = torch.rand((256, 300), device="cuda")
    dip.GaussFIR(x, [2.0], [0], ["mirror"])
    torch.cuda.synchronize()
    n0 = _abi.lib().dipcu_launch_count()
    dip.GaussFIR(x, [2.0], [0], ["mirror"])
    assert _abi.lib().dipcu_launch_count() - n0 == 1
