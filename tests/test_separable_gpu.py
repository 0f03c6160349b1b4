"""dip::SeparableConvolution with real filters of every symmetry and origin, and dip::Uniform with a
rectangular kernel, on the line kernel (general-filter mode, and the uniform filter's running sum in
the reference's operation order), against the oracle (pinned bit-exact to the reference's own
functions in tests/test_oracle_pin.py): random filters, 1D-3D images of several sample types, every
boundary condition, one filter for all axes or one per axis, `process` flags, protected outputs,
and the reference's errors."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from tests.test_gauss_gpu import assert_close, dip

pytestmark = pytest.mark.gpu

SYMS = ["general", "even", "odd", "d-even", "d-odd", "conj", "d-conj"]
BCS = ["mirror", "asym mirror", "periodic", "asym periodic", "add zeros", "zero order", "first order",
       "second order", "third order", "add max", "add min"]


def _random_case(rng):
    nd = int(rng.integers(1, 4))
    shape = tuple(int(v) for v in rng.integers(1, 48, nd))
    dt = [np.float32, np.float64, np.uint16, np.int32, np.uint8][int(rng.integers(0, 5))]
    x = (rng.random(shape) * (1 if dt in (np.float32, np.float64) else 200)).astype(dt)
    nf = 1 if rng.random() < 0.3 else nd
    filters = []
    for _ in range(nf):
        n = int(rng.integers(1, 9))
        sym = SYMS[int(rng.integers(0, len(SYMS)))]
        origin = int(rng.integers(-1, n)) if sym == "general" else -1
        w = rng.standard_normal(n)
        w /= 2 * np.abs(w).sum()                 # gain below 1: rounding errors stay below the range's
        filters.append({"filter": list(w), "origin": origin, "symmetry": sym})
    # "add max" / "add min" pad with +-FLT_MAX, where a different summation order overflows differently
    bcs = [BCS[int(rng.integers(0, len(BCS) - 2))] for _ in range(nd)]
    return x, filters, bcs


def test_random_filters_against_oracle(cuda):
    rng = np.random.default_rng(31)
    for case in range(60):
        x, filters, bcs = _random_case(rng)
        process = None if rng.random() < 0.7 else [bool(v) for v in rng.integers(0, 2, x.ndim)]
        ref = oracle.separable_convolution(x, filters, bcs, process)
        got = dip().SeparableConvolution(x, [dip().OneDimensionalFilter(**f) for f in filters], bcs, process or ())
        assert_close(got, ref, x, f"case {case}: {x.shape} {x.dtype} {[f['symmetry'] for f in filters]} {bcs}")


def test_protected_output_and_long_filter(cuda):
    import torch
    rng = np.random.default_rng(5)
    x = rng.random((60, 70), dtype=np.float32)
    w = rng.standard_normal(100)
    f = {"filter": list(w / (2 * np.abs(w).sum())), "origin": 17, "symmetry": "even"}     # 199 taps
    ref = oracle.separable_convolution(x, [f], ["mirror"])
    assert_close(dip().SeparableConvolution(x, f, ["mirror"]), ref, x, "long even filter")
    xi = (rng.random((40, 50)) * 1000).astype(np.uint16)
    g = {"filter": [1.0, 2.0, 3.0, 2.0], "origin": -1, "symmetry": "general"}
    ref = oracle.separable_convolution(xi, [g], ["periodic"], out_dtype=np.uint16)
    out = torch.zeros((40, 50), dtype=torch.uint16, device="cuda")
    dip().SeparableConvolution(xi, g, ["periodic"], out=out)
    assert int(np.abs(out.cpu().numpy().astype(np.int64) - ref.astype(np.int64)).max()) <= 1


def test_reference_errors(cuda):
    x = np.zeros((10, 10), np.float32)
    with pytest.raises(Exception, match="Symmetry string not recognized"):
        dip().SeparableConvolution(x, {"filter": [1, 2], "symmetry": "sideways"})
    with pytest.raises(Exception, match="Origin outside of filter"):
        dip().SeparableConvolution(x, {"filter": [1, 2, 3], "origin": 3, "symmetry": "general"})
    with pytest.raises(Exception, match="wrong number of elements"):
        dip().SeparableConvolution(x, [{"filter": [1.0]}] * 3)


def test_uniform_against_oracle(cuda):
    rng = np.random.default_rng(8)
    for case in range(40):
        nd = int(rng.integers(1, 4))
        shape = tuple(int(v) for v in rng.integers(1, 60, nd))
        dt = [np.float32, np.float64, np.uint16, np.int32][int(rng.integers(0, 4))]
        x = (rng.random(shape) * (1 if dt in (np.float32, np.float64) else 300)).astype(dt)
        sizes = [int(v) for v in rng.integers(1, 12, nd)]
        bcs = [BCS[int(rng.integers(0, len(BCS)))] for _ in range(nd)]
        ref = oracle.uniform(x, sizes, bcs)
        got = dip().Uniform(x, sizes, bcs)
        assert_close(got, ref, x, f"case {case}: {shape} {x.dtype} {sizes} {bcs}")
        if all(b in ("mirror", "periodic", "add zeros", "zero order") for b in bcs):
            # the same additions in the same order as the reference's running sum: identical samples
            np.testing.assert_array_equal(np.asarray(got), ref, err_msg=f"case {case}")


def test_uniform_large_image_running_sum(cuda):
    rng = np.random.default_rng(9)
    x = rng.random((300, 2000), dtype=np.float32)
    ref = oracle.uniform(x, [31, 5], ["mirror"])
    got = dip().Uniform(x, [31, 5], ["mirror"])
    np.testing.assert_array_equal(np.asarray(got), ref)
