"""dip::GaussIIR (src/linear/gaussiir.cpp): the recursive Gaussian of van Vliet, Young and Verbeek.

CPU: the oracle's restatement (oracle/gauss_oracle.c, or_gauss_iir) is pinned BIT-EXACT to the
reference's own dip::GaussIIR (oracle/_ref) over every recursion order 1-5, derivative order 0-4,
both design methods, sample types and boundary conditions; the reference's own known-answer
checks (gaussiir.cpp:793-876: impulse amplitude and sum, derivatives of x, x^2 and x^3 at the
centre, agreement between recursion orders) are re-run on the oracle.
GPU: the device filter (FP64 scans, one thread per line) against the oracle through the C-ABI:
the bar is the float tolerance 1e-5 x input range; the scans follow the reference's double
operations, so most cases come out bit-identical and the test reports the largest difference.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="the compiled reference (oracle/_ref) is not built")

PIN_CASES = [
    ((64,), [5.0], [0], ["mirror"], (), "discrete time fit", np.float64),
    ((40, 50), [12.0, 3.0], [0, 1], ["periodic", "add zeros"], (), "discrete time fit", np.float32),
    ((40, 50), [12.0, 3.0], [2, 0], ["third order"], (), "forward backward", np.uint16),
    ((20, 30, 25), [2.0, 11.0, 4.0], [1, 2, 3], ["asym mirror", "zero order", "first order"], (), "discrete time fit",
     np.float32),
    ((33, 7), [1.5, 20.0], [4, 0], ["second order", "antisym reflect"], (3, 2), "forward backward", np.int32),
    ((3, 90), [6.0, 0.0], [1, 0], ["asym periodic"], (1,), "discrete time fit", np.uint8),
]


def _input(shape, dt, seed):
    rng = np.random.default_rng(seed)
    if np.issubdtype(dt, np.integer):
        return rng.integers(0, 200, size=shape).astype(dt)
    return (rng.random(shape) * 100.0 - 20.0).astype(dt)


@needs_ref
@pytest.mark.parametrize("case", range(len(PIN_CASES)))
def test_oracle_iir_is_the_reference(case):
    shape, sg, o, bc, fo, dm, dt = PIN_CASES[case]
    x = _input(shape, dt, case)
    got = oracle.gauss_iir(x, sg, o, bc, list(fo) or None, dm)
    ref = oracle.ref_gauss_iir(x, sg, o, bc, fo, dm)
    assert got.dtype == ref.dtype
    assert np.array_equal(got, ref), float(np.abs(got.astype(np.float64) - ref).max())


@needs_ref
def test_oracle_iir_every_design_is_the_reference():
    """Recursion orders 1-5 x derivative orders 0-4 x both design methods, on a short line with a
    border longer than the line (multiple reflections), bit for bit."""
    x = _input((23,), np.float64, 7)
    for nn in range(1, 6):
        for order in range(5):
            for dm in ("discrete time fit", "forward backward"):
                got = oracle.gauss_iir(x, [9.0], [order], ["mirror"], [nn], dm)
                ref = oracle.ref_gauss_iir(x, [9.0], [order], ["mirror"], [nn], dm)
                assert np.array_equal(got, ref), (nn, order, dm)


@needs_ref
def test_oracle_iir_add_max_is_the_reference():
    """"add max" pads with the largest double; the reference's scans turn that into NaNs, in the
    same places."""
    x = _input((12, 30), np.float32, 3)
    got = oracle.gauss_iir(x, [4.0], [0], ["add max"])
    ref = oracle.ref_gauss_iir(x, [4.0], [0], ["add max"])
    assert np.array_equal(got, ref, equal_nan=True)


def test_reference_known_answers_on_the_oracle():
    """gaussiir.cpp:793-876, re-run on the oracle: an impulse gives the normalised Gaussian's peak
    and sums to 1; recursion orders agree within the reference's bounds; derivatives of x, x^2
    and x^3 at the centre are 1, 2 and 6."""
    img = np.zeros(256)
    img[128] = 1.0
    sigma = 5.0
    amplitude = 1.0 / (np.sqrt(2.0 * np.pi) * sigma)
    r1 = oracle.gauss_iir(img, [sigma], [0], [], [5], "discrete time fit")
    assert abs(r1[128] - amplitude) < 0.00015
    assert abs(r1.sum() - 1.0) < 1e-6
    for fo, dm, tol in ((4, "discrete time fit", 0.0003), (3, "discrete time fit", 0.002), (2, "discrete time fit", 0.004),
                        (5, "forward backward", 0.003), (4, "forward backward", 0.002), (3, "forward backward", 0.009)):
        r2 = oracle.gauss_iir(img, [sigma], [0], [], [fo], dm)
        assert np.abs(r1 - r2).max() <= tol, (fo, dm)
    ramp = np.arange(-128.0, 128.0)
    for order, img2, want, fos in ((1, ramp, 1.0, (5, 4, 3)), (2, ramp * ramp, 2.0, (5, 4, 3)),
                                   (3, ramp * ramp * ramp, 6.0, (5, 4))):
        for fo in fos:
            for dm in ("discrete time fit", "forward backward"):
                r = oracle.gauss_iir(img2, [sigma], [order], [], [fo], dm)
                assert r[128] == pytest.approx(want, rel=1e-5), (order, fo, dm)


GPU_CASES = PIN_CASES + [
    ((48, 64, 80), [15.0, 12.0, 11.0], [0, 0, 0], ["mirror"], (), "discrete time fit", np.float32),
    ((300, 257), [25.0, 10.5], [1, 2], ["periodic", "mirror"], (), "discrete time fit", np.float32),
    ((17, 19, 5, 6), [3.0, 4.0, 5.0, 6.0], [0, 1, 0, 2], ["mirror", "add zeros", "add min", "zero order"], (),
     "forward backward", np.float64),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(GPU_CASES)))
def test_gauss_iir_matches_oracle(cuda, case):
    import diplib_b200 as dip
    shape, sg, o, bc, fo, dm, dt = GPU_CASES[case]
    x = _input(shape, dt, 100 + case)
    got = dip.GaussIIR(x, sg, o, bc, list(fo), dm)
    ref = oracle.gauss_iir(x, sg, o, bc, list(fo) or None, dm)
    assert got.dtype == ref.dtype and got.shape == ref.shape
    fin = np.isfinite(ref)
    assert np.array_equal(np.isfinite(got), fin)
    tol = 1e-5 * max(1.0, float(x.max()) - float(x.min()))
    err = float(np.abs(got[fin].astype(np.float64) - ref[fin]).max()) if fin.any() else 0.0
    print(f"GaussIIR {shape} {dt.__name__} {sg} {o} {dm}: max |GPU - oracle| = {err:.3g}"
          f"{' (bit-identical)' if np.array_equal(got, ref, equal_nan=True) else ''}")
    assert err <= tol


@pytest.mark.gpu
def test_gauss_iir_through_the_c_abi_with_strides_and_protected_output(cuda):
    """A strided view in, a protected uint16 output (clamp_cast on the write), through the C-ABI."""
    import torch

    from diplib_b200 import _abi
    from diplib_b200.filtering import BoundaryConditionFromString, image_desc
    base = _input((60, 90), np.float32, 5) * 20.0
    x = np.ascontiguousarray(base)[::2, 1::3]
    xt = torch.from_numpy(np.ascontiguousarray(base)).cuda()[::2, 1::3]
    out = torch.empty(x.shape, dtype=torch.uint16, device="cuda")
    sg, o = [14.0, 3.0], [0, 0]
    bcs = [BoundaryConditionFromString("mirror")] * 2
    st = _abi.lib().dipcu_gauss_iir(ctypes.byref(image_desc(xt)), ctypes.byref(image_desc(out)),
                                    (ctypes.c_double * 2)(*sg), (ctypes.c_uint32 * 2)(*o), (ctypes.c_int32 * 2)(*bcs),
                                    None, _abi.IIR_DISCRETE_TIME_FIT, 3.0, None)
    assert st == 0, _abi.last_error()
    torch.cuda.synchronize()
    ref = oracle.gauss_iir(x, sg, o, ["mirror"], None, "discrete time fit", out_dtype=np.uint16)
    got = out.cpu().numpy()
    assert np.abs(got.astype(np.int64) - ref.astype(np.int64)).max() <= 1
    # errors as the reference raises them
    with pytest.raises(Exception, match="Invalid flag"):
        import diplib_b200 as dip
        dip.GaussIIR(x, [3.0], [0], [], [], "bogus")
    assert _abi.lib().dipcu_gauss_iir(ctypes.byref(image_desc(xt)), ctypes.byref(image_desc(out)),
                                      (ctypes.c_double * 2)(*sg), (ctypes.c_uint32 * 2)(5, 0),
                                      (ctypes.c_int32 * 2)(*bcs), None, 0, 3.0, None) == _abi.ERR_INVALID_ARG


def test_oracle_iir_matches_golden_fixtures():
    """The restatement against fixtures generated from the compiled dip::GaussIIR
    (tests/golden/make_golden.py): bit-exact, with no reference tree needed."""
    import os

    from tests.golden.make_golden import IIR_CASES, make_input
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "gauss_iir_ref.npz"))
    for name, seed, shape, dtype, sig, ords, bcs, fo, dm in IIR_CASES:
        x = make_input(seed, shape, dtype)
        got = oracle.gauss_iir(x, sig, ords, bcs, fo or None, dm)
        assert got.dtype == ref[name].dtype, name
        assert np.array_equal(got, ref[name], equal_nan=True), (name, float(np.nanmax(np.abs(got - ref[name]))))


@pytest.mark.gpu
def test_gauss_iir_device_matches_golden_fixtures(cuda):
    """The device filter against the reference's own outputs (golden fixtures), at the float bar."""
    import os

    import diplib_b200 as dip
    from tests.golden.make_golden import IIR_CASES, make_input
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "gauss_iir_ref.npz"))
    for name, seed, shape, dtype, sig, ords, bcs, fo, dm in IIR_CASES:
        x = make_input(seed, shape, dtype)
        got = dip.GaussIIR(x, sig, ords, bcs, fo, dm)
        tol = 1e-5 * max(1.0, float(x.max()) - float(x.min()))
        assert got.dtype == ref[name].dtype and np.abs(got.astype(np.float64) - ref[name]).max() <= tol, name
