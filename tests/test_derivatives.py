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


MULTI_CASES = [
    # (shape, sigmas, boundary conditions, dtype): all taken by the multi-output tile kernel
    ((96, 131), [1.5], ["mirror"], np.float32),
    ((37, 50, 70), [1.0, 2.0, 0.8], ["periodic", "add zeros", "asym mirror"], np.float32),
    ((24, 33, 45), [1.0, 1.5, 2.0], ["mirror"], np.uint16),
    ((19, 1, 40), [2.0, 1.0, 1.5], ["zero order", "asym periodic", "mirror"], np.float32),
    ((70, 9), [0.8, 2.0], ["mirror"], np.uint8),
]


def _launches():
    from diplib_b200 import _abi
    return int(_abi.lib().dipcu_launch_count())


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(MULTI_CASES)))
def test_multi_output_kernel_matches_oracle(cuda, case, monkeypatch):
    """Gradient, Hessian, Laplace and GradientMagnitude each from ONE launch of the multi-output
    tile kernel (counted by the library's launch counter), against the oracle's compositions of
    the restated GaussFIR (pinned bit-exact to the reference's own functions above)."""
    import torch

    import diplib_b200 as dip
    from diplib_b200 import derivatives
    monkeypatch.setattr(derivatives, "USE_MULTI_OUTPUT", True)
    shape, sg, bc, dt = MULTI_CASES[case]
    x = _input(shape, dt, 80 + case)
    xt = x                      # numpy in: staged to the device by the function, numpy out
    tol = 1e-5 * max(1.0, float(x.max()) - float(x.min()))
    for fn, ref in ((dip.Gradient, oracle.gradient(x, sg, bc, 3.0)),
                    (dip.Hessian, oracle.hessian(x, sg, bc, 3.0)),
                    (dip.Laplace, oracle.laplace(x, sg, bc, 3.0))):
        n0 = _launches()
        got = fn(xt, sg, "best", bc)
        torch.cuda.synchronize()
        assert _launches() - n0 == 1, fn.__name__
        assert got.shape == ref.shape and np.abs(got - ref).max() <= tol, (fn.__name__, float(np.abs(got - ref).max()))
    g = oracle.gradient(x, sg, bc, 3.0)
    n0 = _launches()
    got = dip.GradientMagnitude(xt, sg, "best", bc)
    torch.cuda.synchronize()
    ref = np.sqrt((g.astype(np.float64) ** 2).sum(axis=0))
    if g.shape[0] > 1:
        assert _launches() - n0 == 1
    assert np.abs(got - ref).max() <= tol


@pytest.mark.gpu
def test_multi_output_products_through_the_c_abi(cuda):
    """Mode 1 (dip::StructureTensor's products g_i g_j, DIPlib's symmetric-matrix order) and
    protected integer outputs (clamp_cast on the write), called through the C-ABI."""
    import ctypes

    import torch

    from diplib_b200 import _abi
    from diplib_b200.filtering import BoundaryConditionFromString, image_desc
    x = _input((30, 41, 67), np.float32, 7)
    sg, bc = [1.0, 1.2, 0.9], ["mirror", "periodic", "add zeros"]
    g = oracle.gradient(x, sg, bc, 3.0).astype(np.float64)
    pairs = oracle.symmetric_pairs(3)
    ref = np.stack([g[i] * g[j] for i, j in pairs])
    xt = torch.from_numpy(x).cuda()
    outs = [torch.empty(x.shape, dtype=torch.float32, device="cuda") for _ in pairs]
    orders = [1, 0, 0, 0, 1, 0, 0, 0, 1]
    bcs = [BoundaryConditionFromString(b) for b in bc]
    lib = _abi.lib()
    din = image_desc(xt)
    douts = (_abi.ImageDesc * 6)(*[image_desc(o) for o in outs])
    st = lib.dipcu_gauss_fir_multi(ctypes.byref(din), douts, 6, (ctypes.c_uint32 * 9)(*orders), 3, 1,
                                   (ctypes.c_double * 3)(*sg), (ctypes.c_int32 * 3)(*bcs), 3.0, None)
    assert st == 0, _abi.last_error()
    torch.cuda.synchronize()
    got = np.stack([o.cpu().numpy() for o in outs])
    scale = float(np.abs(ref).max())
    assert np.abs(got - ref).max() <= 1e-5 * scale
    # wrong output count for the mode, and a case the kernel does not take (half-width > 8)
    assert lib.dipcu_gauss_fir_multi(ctypes.byref(din), douts, 5, (ctypes.c_uint32 * 9)(*orders), 3, 1,
                                     (ctypes.c_double * 3)(*sg), (ctypes.c_int32 * 3)(*bcs), 3.0, None) == _abi.ERR_INVALID_ARG
    big = (ctypes.c_double * 3)(4.0, 4.0, 4.0)
    assert lib.dipcu_gauss_fir_multi_supported(ctypes.byref(din), (ctypes.c_uint32 * 9)(*orders), 3, big,
                                               (ctypes.c_int32 * 3)(*bcs), 3.0) == 0
    # unsigned 8-bit outputs of the gradient components: clamped and rounded like dip::clamp_cast
    o8 = [torch.empty(x.shape, dtype=torch.uint8, device="cuda") for _ in range(3)]
    x8 = (x * 400.0).astype(np.float32)
    xt8 = torch.from_numpy(x8).cuda()
    d8 = (_abi.ImageDesc * 3)(*[image_desc(o) for o in o8])
    st = lib.dipcu_gauss_fir_multi(ctypes.byref(image_desc(xt8)), d8, 3, (ctypes.c_uint32 * 9)(*orders), 3, 0,
                                   (ctypes.c_double * 3)(*sg), (ctypes.c_int32 * 3)(*bcs), 3.0, None)
    assert st == 0, _abi.last_error()
    torch.cuda.synchronize()
    g8 = oracle.gradient(x8, sg, bc, 3.0).astype(np.float64)
    ref8 = np.clip(np.round(g8), 0, 255)
    got8 = np.stack([o.cpu().numpy() for o in o8]).astype(np.float64)
    assert np.abs(got8 - ref8).max() <= 1


@pytest.mark.gpu
def test_derivatives_fall_back_per_component_beyond_the_multi_kernel(cuda, monkeypatch):
    """Half-widths above 8 (sigma 4): the multi-output kernel declines and every component is its
    own GaussFIR call, still against the oracle."""
    import torch

    import diplib_b200 as dip
    from diplib_b200 import derivatives
    monkeypatch.setattr(derivatives, "USE_MULTI_OUTPUT", True)
    x = _input((40, 52), np.float32, 3)
    xt = torch.from_numpy(x).cuda()
    n0 = _launches()
    got = dip.Hessian(xt, [4.0], "best", ["mirror"])
    torch.cuda.synchronize()
    assert _launches() - n0 >= 3
    ref = oracle.hessian(x, [4.0], ["mirror"], 3.0)
    assert np.abs(got.cpu().numpy() - ref).max() <= 1e-5
