"""Pins the C restatement of the Gaussian FIR path (oracle/gauss_oracle.c) to the reference:
bit-exact against fixtures generated from the compiled DIPlib sources (tests/golden/), against
the live reference library where it is present, and on the known-answer properties of
DIPlib's own Gaussian tests (src/linear/gauss.cpp:496-540)."""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle
from tests.golden.make_golden import CASES, make_input

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_gauss_matches_reference_fixtures():
    ref = np.load(os.path.join(GOLDEN, "gauss_ref.npz"))
    for name, seed, shape, dtype, sig, ords, bcs, trunc in CASES:
        x = make_input(seed, shape, dtype)
        y = oracle.gauss_fir(x, sig, ords, bcs or ["mirror"], trunc)
        assert y.dtype == ref[name].dtype, name
        assert np.array_equal(y, ref[name], equal_nan=True), name


def test_half_gaussian_matches_reference_fixtures():
    ref = np.load(os.path.join(GOLDEN, "half_gaussian_ref.npz"))
    for key in ref.files:
        s, o, d = key[1:].split("_")
        got = oracle.half_gaussian(float(s), int(o[1:]), 3.0, bool(int(d[1:])))
        assert np.array_equal(got, ref[key]), key


def test_expand_buffer_matches_reference_fixtures():
    ref = np.load(os.path.join(GOLDEN, "expand_buffer_ref.npz"))
    for key in ref.files:
        if not key.endswith("|in"):
            continue
        bc, n, left, right, _ = key.split("|")
        got = oracle.expand_buffer(ref[key], int(left), int(right), bc)
        assert np.array_equal(got, ref[key[:-3] + "|out"]), key


def test_structure_tensor_matches_reference_fixture():
    ref = np.load(os.path.join(GOLDEN, "structure_tensor_ref.npz"))["st"]
    x = make_input(21, (10, 12, 14), "float32")
    got = oracle.structure_tensor(x, 1.0, 2.0, "mirror", 3.0)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-6 * np.abs(ref).max())


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_gauss_matches_live_reference_fuzz():
    rng = np.random.default_rng(1234)
    bcs = ["mirror", "asym mirror", "antisym reflect", "periodic", "asym periodic", "add zeros", "zero order",
           "first order", "second order", "third order"]
    for it in range(60):
        nd = int(rng.integers(1, 4))
        shape = tuple(int(rng.integers(1, 24)) for _ in range(nd))
        dtype = [np.float32, np.uint16, np.uint8, np.int16, np.float64, np.int32][int(rng.integers(0, 6))]
        x = make_input(int(rng.integers(0, 1 << 30)), shape, dtype)
        sig = [float(rng.choice([0.0, 0.6, 1.0, 1.7, 2.5, 4.0])) for _ in range(nd)]
        ords = [int(rng.integers(0, 4)) for _ in range(nd)]
        bc = [str(rng.choice(bcs)) for _ in range(nd)]
        tr = float(rng.choice([2.0, 3.0, 4.5]))
        a = oracle.gauss_fir(x, sig, ords, bc, tr)
        b = oracle.ref_gauss(x, sig, ords, bc, tr)
        assert np.array_equal(a, b, equal_nan=True), (it, shape, dtype, sig, ords, bc, tr)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_protected_output_matches_live_reference():
    x = make_input(5, (30, 40), np.float32) * 300.0
    for out_dt in (np.uint8, np.int16, np.float64):
        a = oracle.gauss_fir(x, [2.0], [0], ["mirror"], 3.0, out_dtype=out_dt)
        b = oracle.ref_gauss(x, [2.0], [0], ["mirror"], 3.0, out_dtype=out_dt)
        assert np.array_equal(a, b), out_dt


def test_known_answers_from_reference_tests():
    # src/linear/gauss.cpp:496-540: delta at 128 of a 256-sample dfloat line, sigma 5.
    img = np.zeros(256, np.float64)
    img[128] = 1.0
    fir = oracle.gauss_fir(img, [5.0], [0])
    assert abs(fir.sum() - 1.0) < 1e-12
    # The reference bounds FT vs the amplitude by 0.00015 and FIR vs FT by 0.0006.
    assert abs(fir[128] - 1.0 / (np.sqrt(2 * np.pi) * 5.0)) < 0.00015 + 0.0006
    ramp = np.arange(-128, 128, dtype=np.float64)
    assert fir.dtype == np.float64
    assert oracle.gauss_fir(ramp, [5.0], [1])[128] == pytest.approx(1.0)
    assert oracle.gauss_fir(ramp * ramp, [5.0], [2])[128] == pytest.approx(2.0)


def test_order_gt_3_rejected():
    with pytest.raises(ValueError, match="order > 3"):
        oracle.gauss_fir(np.zeros((8, 8), np.float32), [1.0], [4])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_structure_tensor_matches_live_reference():
    """Size-1 axes drop out of the gradient (FindGradientDimensions); integer inputs go through
    the flex type; every index-mapping boundary condition."""
    rng = np.random.default_rng(77)
    cases = [((9, 11), np.float32, 1.0, 2.0, "mirror"), ((1, 12, 13), np.float32, 1.0, 3.0, "periodic"),
             ((7, 1, 10), np.uint16, 1.5, 2.0, "add zeros"), ((6, 8, 9), np.int32, 0.9, 1.5, "asym mirror"),
             ((5, 9, 7), np.float64, 1.0, 2.5, "zero order"), ((17,), np.float32, 1.0, 2.0, "first order")]
    for shape, dt, gsig, tsig, bc in cases:
        x = (rng.random(shape) * 1000).astype(dt)
        ref = oracle.ref_structure_tensor(x, gsig, tsig, bc, 3.0)
        got = oracle.structure_tensor(x, gsig, tsig, bc, 3.0)
        assert got.shape == ref.shape and got.dtype == ref.dtype, (shape, got.shape, ref.shape)
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-6 * np.abs(ref).max(), err_msg=str((shape, bc)))


@pytest.mark.skipif(not oracle.ref_available(), reason="the compiled reference (oracle/_ref) is not built")
def test_reference_one_thread_equals_all_threads():
    """The reference's own multithreading check (src/linear/gauss.cpp:547-569): dip::Gauss with
    sigma 2 of a 256 x 192 x 59 dfloat noise volume gives the same samples with one thread and
    with all of them -- the configuration the bench's reference arm runs in."""
    x = np.random.default_rng(0).standard_normal((59, 192, 256))
    try:
        oracle.ref_set_threads(1)
        one = oracle.ref_gauss(x, [2.0], [0], None, 3.0)
        oracle.ref_set_threads(0)
        many = oracle.ref_gauss(x, [2.0], [0], None, 3.0)
    finally:
        oracle.ref_set_threads(0)
    assert np.array_equal(one, many)


def test_separable_convolution_and_uniform_pinned_to_the_reference():
    """The oracle's general SeparableConvolution (every real symmetry, origins, one or per-axis
    filters, process flags) and rectangular Uniform (running sum) equal the reference's own
    dip::SeparableConvolution / dip::Uniform bit for bit."""
    if not oracle.ref_available():
        pytest.skip("reference build not present")
    rng = np.random.default_rng(44)
    syms = ["general", "even", "odd", "d-even", "d-odd", "conj", "d-conj"]
    bcs_all = ["mirror", "asym mirror", "periodic", "asym periodic", "add zeros", "add max", "add min", "zero order",
               "first order", "second order", "third order"]
    for case in range(50):
        nd = int(rng.integers(1, 4))
        shape = tuple(int(v) for v in rng.integers(1, 30, nd))
        dt = [np.float32, np.float64, np.uint16, np.int32, np.uint8][int(rng.integers(0, 5))]
        x = (rng.random(shape) * 100).astype(dt)
        nf = 1 if rng.random() < 0.3 else nd
        filters = []
        for _ in range(nf):
            n = int(rng.integers(1, 8))
            sym = syms[int(rng.integers(0, len(syms)))]
            filters.append({"filter": list(rng.standard_normal(n)),
                            "origin": int(rng.integers(-1, n)) if sym == "general" else -1, "symmetry": sym})
        bcs = [bcs_all[int(rng.integers(0, len(bcs_all)))] for _ in range(nd)]
        process = None if rng.random() < 0.7 else [bool(v) for v in rng.integers(0, 2, nd)]
        ref = oracle.ref_separable_convolution(x, filters, bcs, process)
        got = oracle.separable_convolution(x, filters, bcs, process)
        np.testing.assert_array_equal(got, ref, err_msg=f"separable case {case}")
        sizes = [int(v) for v in rng.integers(1, 10, nd)]
        np.testing.assert_array_equal(oracle.uniform(x, sizes, bcs), oracle.ref_uniform(x, sizes, bcs),
                                      err_msg=f"uniform case {case}")


def test_gauss_ft_pinned_to_the_reference():
    """The oracle's dip::GaussFT restatement (boundary extension to a 5-smooth DFT size, centred
    transform, the Gaussian look-up table, real inverse, crop) equals the reference's
    dip::Gauss(method "FT") to float rounding, for even and odd transform sizes (the odd sizes
    exercise the reference's half-line shift, which swaps the outermost frequency planes along
    its real-to-complex dimension)."""
    if not oracle.ref_available():
        pytest.skip("reference build not present")
    rng = np.random.default_rng(12)
    cases = [((40,), [0.5], [0], ["mirror"]), ((41,), [0.5], [0], ["periodic"]), ((38,), [1.0], [1], ["mirror"]),
             ((40, 50), [0.5, 0.6], [0, 0], ["mirror"]), ((21, 30, 17), [0.6, 2.0, 0.6], [0, 1, 2], ["periodic"]),
             ((64,), [0.4], [5], ["add zeros"]), ((31, 28), [1.0, 0.5], [2, 3], ["mirror"]),
             ((33, 41), [0.7, 0.5], [1, 4], ["zero order"]), ((40, 40), [0.5, 0.5], [1, 1], ["mirror"]),
             ((9, 40, 7), [0.5, 0.5, 0.5], [1, 0, 1], ["asym mirror"]), ((41, 2), [0.5, 0.5], [0, 1], ["mirror"]),
             ((43, 43), [0.5, 1.5], [1, 2], ["mirror", "periodic"])]
    for shape, sig, o, bcs in cases:
        x = rng.random(shape).astype(np.float32)
        ref = oracle.ref_gauss(x, sig, o, bcs, 3.0, method="FT")
        got = oracle.gauss_ft(x, sig, o, 3.0, bcs)
        assert ref.dtype == np.float32
        err = np.abs(ref.astype(np.float64) - got).max() / max(1.0, float(np.abs(ref).max()))
        assert err < 2e-6, (shape, sig, o, bcs, err)
    x = rng.random((40, 33))
    ref = oracle.ref_gauss(x, [0.5, 0.5], [1, 0], ["mirror"], 3.0, method="FT")
    np.testing.assert_allclose(oracle.gauss_ft(x, [0.5, 0.5], [1, 0], 3.0, ["mirror"]), ref, rtol=0, atol=1e-13)
