"""dip::GaussFT on the device (cuFFT transforms, gather / spectrum / scatter kernels) against the
oracle's restatement, which tests/test_oracle_pin.py pins to the reference's dip::Gauss "FT":
1D-3D images, even and odd transform lengths (the odd ones exercise the reference's swapped
outermost frequency planes), derivative orders above 3, every boundary condition the extension
takes, no extension, float / integer / double inputs, a strided input that moves the reference's
real-to-complex axis, and dip::Gauss's method dispatch."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from tests.test_gauss_gpu import dip, to_dev

pytestmark = pytest.mark.gpu


def _close(got, ref, what):
    got = np.asarray(got)
    assert got.shape == ref.shape and got.dtype == ref.dtype, what
    scale = max(1.0, float(np.abs(ref).max()))
    tol = (2e-5 if ref.dtype == np.float32 else 1e-11) * scale
    err = float(np.abs(got.astype(np.float64) - ref.astype(np.float64)).max())
    assert err <= tol, f"{what}: max err {err} > {tol}"


CASES = [
    ((40,), [0.5], [0], ["mirror"]),
    ((41,), [0.5], [0], ["periodic"]),
    ((38,), [1.0], [1], ["mirror"]),
    ((64,), [0.4], [5], ["add zeros"]),
    ((40, 50), [0.5, 0.6], [0, 0], ["mirror"]),
    ((31, 28), [1.0, 0.5], [2, 3], ["mirror"]),
    ((33, 41), [0.7, 0.5], [1, 4], ["zero order"]),
    ((43, 43), [0.5, 1.5], [1, 2], ["mirror", "periodic"]),
    ((41, 2), [0.5, 0.5], [0, 1], ["mirror"]),
    ((9, 40, 7), [0.5, 0.5, 0.5], [1, 0, 1], ["asym mirror"]),
    ((21, 30, 17), [0.6, 2.0, 0.6], [0, 1, 2], ["periodic"]),
    ((16, 33, 25), [0.3, 0.7, 1.2], [0, 0, 0], ["asym periodic"]),
    ((200, 300), [2.0, 2.0], [0, 0], ["mirror"]),
]


@pytest.mark.parametrize("case", CASES, ids=[str(c[0]) + "-" + str(c[2]) + "-" + c[3][0] for c in CASES])
def test_against_oracle(cuda, case):
    shape, sig, o, bcs = case
    rng = np.random.default_rng(sum(shape))
    x = rng.random(shape).astype(np.float32)
    ref = oracle.gauss_ft(x, sig, o, 3.0, bcs)
    _close(dip().GaussFT(x, sig, o, 3.0, "spatial", "spatial", bcs), ref, str(case))


@pytest.mark.parametrize("dt", [np.uint16, np.uint8, np.int32, np.float64])
def test_input_types(cuda, dt):
    rng = np.random.default_rng(3)
    x = (rng.random((27, 35)) * 200).astype(dt)
    ref = oracle.gauss_ft(x, [0.6, 1.1], [1, 0], 3.0, ["mirror"])
    assert ref.dtype == (np.float64 if dt in (np.int32, np.float64) else np.float32)
    _close(dip().GaussFT(x, [0.6, 1.1], [1, 0], 3.0, "spatial", "spatial", ["mirror"]), ref, str(dt))


def test_without_extension(cuda):
    rng = np.random.default_rng(5)
    for shape in [(45,), (30, 45), (9, 21, 15)]:
        x = rng.random(shape).astype(np.float32)
        nd = len(shape)
        ref = oracle.gauss_ft(x, [0.7] * nd, [1] + [0] * (nd - 1), 3.0, None)
        _close(dip().GaussFT(x, [0.7] * nd, [1] + [0] * (nd - 1), 3.0), ref, str(shape))


def test_strided_input_moves_the_real_to_complex_axis(cuda):
    """Without extension the reference transforms its real-to-complex axis along the smallest
    input stride: a transposed view makes that the second axis."""
    rng = np.random.default_rng(9)
    base = rng.random((35, 45)).astype(np.float32)          # numpy (y, x): x has 45 samples
    view = to_dev(base).t()                                  # (45, 35): x now has stride 35
    xs = np.ascontiguousarray(base.T)
    ref = oracle.gauss_ft(xs, [0.6, 0.9], [0, 1], 3.0, None, rdim=1)
    _close(dip().GaussFT(view, [0.6, 0.9], [0, 1], 3.0).cpu().numpy(), ref, "transposed")


def test_gauss_dispatch_and_protected_output(cuda):
    rng = np.random.default_rng(11)
    x = rng.random((50, 61)).astype(np.float32)
    ref = oracle.gauss_ft(x, [0.5, 0.5], [0, 0], 3.0, ["mirror"])   # "best" picks FT for sigma < 0.8
    _close(dip().Gauss(x, [0.5, 0.5], [0, 0], "best"), ref, "best")
    _close(dip().Gauss(x, [0.5, 0.5], [0, 0], "gaussFT", ["periodic"]), oracle.gauss_ft(x, [0.5, 0.5], [0, 0], 3.0, ["periodic"]),
           "gaussFT")
    out = torch.zeros((50, 61), dtype=torch.float64, device="cuda")
    dip().GaussFT(x, [1.0, 1.0], [0, 1], 3.0, "spatial", "spatial", ["mirror"], out=out)
    _close(out.cpu().numpy().astype(np.float32), oracle.gauss_ft(x, [1.0, 1.0], [0, 1], 3.0, ["mirror"]), "out float64")
    same = dip().GaussFT(x, [0.0, -1.0], [0, 0], 3.0)                # nothing to do: a converted copy
    np.testing.assert_array_equal(same, x)


def test_errors(cuda):
    x = np.zeros((4, 5, 6, 7), np.float32)
    with pytest.raises(Exception, match="up to 3 dimensions"):
        dip().GaussFT(x, [1.0], [0])
    with pytest.raises(Exception, match="boundary extension"):
        dip().GaussFT(np.zeros((10, 10), np.float32), [1.0], [0], 3.0, "spatial", "spatial", ["first order"])
