"""dip::Gradient / GradientMagnitude / Hessian / Laplace (src/linear/derivative.cpp:120-418) on the
Gaussian FIR path: every component against the oracle's composition of the restated GaussFIR
(max abs error 1e-5 times the input range), and on the CPU the axis selection and DIPlib's
symmetric-matrix component order."""
from __future__ import annotations

import numpy as np
import pytest

import oracle


def test_find_gradient_dimensions_host_logic():
    from diplib_b200.derivatives import find_gradient_dimensions
    # numpy shape (z, y, x) = (1, 5, 7): DIPlib axes x=0, y=1, z=2; z has size 1.
    assert find_gradient_dimensions((1, 5, 7), [1.0])[0] == [0, 1]
    assert find_gradient_dimensions((4, 5, 7), [1.0, 0.0, 2.0])[0] == [0, 2]
    assert find_gradient_dimensions((4, 5, 7), [1.0], process=[False, True, True])[0] == [1, 2]
    assert find_gradient_dimensions((4, 5, 7), 2.0)[1] == [2.0, 2.0, 2.0]


def test_symmetric_matrix_order_is_column_wise():
    # include/diplib/library/tensor.h:100-110: diagonal, then above it column by column.
    assert oracle.symmetric_pairs(3) == [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    assert oracle.symmetric_pairs(4) == [(0, 0), (1, 1), (2, 2), (3, 3), (0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (2, 3)]


CASES = [
    ((96, 131), [1.5], ["mirror"], np.float32, None),
    ((40, 1, 70), [1.0, 2.0, 0.8], ["periodic", "add zeros", "asym mirror"], np.float32, None),
    ((24, 33, 45), [1.0, 1.5, 2.0], ["mirror"], np.uint16, None),
    ((30, 40, 50), [2.0], ["zero order"], np.float32, [True, False, True]),
    ((2, 20, 30, 25), [1.0], ["mirror"], np.float32, None),
]


def _input(shape, dt, seed):
    rng = np.random.default_rng(seed)
    if dt == np.uint16:
        return rng.integers(0, 4096, size=shape, dtype=np.uint16)
    return (rng.random(shape, dtype=np.float32) - 0.5).astype(dt)


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(CASES)))
def test_derivatives_match_oracle(cuda, case):
    import diplib_b200 as dip
    shape, sg, bc, dt, process = CASES[case]
    x = _input(shape, dt, 40 + case)
    rng = float(x.max()) - float(x.min())
    tol = 1e-5 * max(1.0, rng)
    pr = process if process is not None else ()
    got = dip.Gradient(x, sg, "best", bc, pr)
    ref = oracle.gradient(x, sg, bc, 3.0, process)
    assert got.shape == ref.shape and np.abs(got - ref).max() <= tol
    got = dip.Hessian(x, sg, "gauss", bc, pr)
    ref = oracle.hessian(x, sg, bc, 3.0, process)
    assert got.shape == ref.shape and np.abs(got - ref).max() <= tol
    got = dip.Laplace(x, sg, "best", bc, pr)
    ref = oracle.laplace(x, sg, bc, 3.0, process)
    assert got.shape == ref.shape and np.abs(got - ref).max() <= tol
    got = dip.GradientMagnitude(x, sg, "best", bc, pr)
    g = oracle.gradient(x, sg, bc, 3.0, process)
    ref = np.sqrt((g.astype(np.float64) ** 2).sum(axis=0)).astype(g.dtype)
    assert got.shape == ref.shape and np.abs(got - ref).max() <= tol


@pytest.mark.gpu
def test_derivatives_reject_what_the_fir_path_does_not_take(cuda):
    import diplib_b200 as dip
    x = np.zeros((8, 8), np.float32)
    with pytest.raises(NotImplementedError):
        dip.Hessian(x, [1.0], "finitediff")
    with pytest.raises(dip.ParameterError):
        dip.Gradient(x, [0.0])          # no axis with sigma > 0: DIPlib's E::DIMENSIONALITY_NOT_SUPPORTED


@pytest.mark.skipif(not oracle.ref_available(), reason="the compiled reference (oracle/_ref) is not built")
@pytest.mark.parametrize("case", range(len(CASES)))
def test_oracle_compositions_are_the_reference(case):
    """Pins the oracle's compositions to the reference's own dip::Gradient / GradientMagnitude /
    Hessian / Laplace (oracle/_ref): bit-exact for the first three (the same GaussFIR calls in
    the same order, the Hessian's components in the same storage order), within float rounding
    for the magnitude, which this test forms in double."""
    shape, sg, bc, dt, _ = CASES[case]
    x = _input(shape, dt, 60 + case)
    for which, fn in (("gradient", oracle.gradient), ("hessian", oracle.hessian), ("laplace", oracle.laplace)):
        ref = oracle.ref_derivative_op(which, x, sg, bc)
        got = fn(x, sg, bc, 3.0)
        assert ref.shape == got.shape and ref.dtype == got.dtype, which
        assert np.array_equal(ref, got), (which, float(np.abs(ref - got).max()))
    ref = oracle.ref_derivative_op("gradient_magnitude", x, sg, bc)
    g = oracle.gradient(x, sg, bc, 3.0).astype(np.float64)
    assert np.abs(ref - np.sqrt((g ** 2).sum(axis=0))).max() <= 1e-6 * max(1.0, float(np.abs(ref).max()))
