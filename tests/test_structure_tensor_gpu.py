"""Structure tensor (dipcu_structure_tensor / dipcu_structure_tensor_backward) against the oracle.

Forward: the reference fixture (tests/golden/structure_tensor_ref.npz), the oracle's restatement
of dip::StructureTensor on 1D-3D inputs of several types, boundary conditions and size-1 axes,
DIPlib's interleaved layout (component stride 1) through the C-ABI, and one volume of the
differentiable-structure-tensor workload (192^3 sfloat, gradient sigma 1, tensor sigma 4, mirror).
The bar is a max abs error of 1e-5 times the largest component magnitude.

Backward: FP64 central finite differences of L = sum_c <W_c, T_c> on small volumes; at full size
the degree-2 homogeneity of T (T(a x) = a^2 T(x)), which gives <dL/dx, x> = 2 L exactly for every
linear boundary condition.
"""
from __future__ import annotations

import ctypes
import os
import zlib

import numpy as np
import pytest
import torch

import oracle
from tests.golden.make_golden import make_input

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def st_gpu(x: np.ndarray, gsig, tsig, bc="mirror", trunc=3.0) -> np.ndarray:
    import diplib_b200 as dip
    return dip.StructureTensor(x, None, gsig, tsig, "gaussFIR", bc, trunc)


def smoothed_noise(seed: int, shape) -> np.ndarray:
    """N(0,1) noise smoothed by a Gaussian of sigma 2 (the workload's input distribution)."""
    rng = np.random.default_rng(seed)
    n = rng.standard_normal(shape).astype(np.float32)
    return oracle.gauss_fir(n, [2.0] * len(shape), [0] * len(shape), ["mirror"], 3.0)


def test_forward_matches_reference_fixture(cuda):
    ref = np.load(os.path.join(GOLDEN, "structure_tensor_ref.npz"))["st"]
    x = make_input(21, (10, 12, 14), "float32")
    got = st_gpu(x, 1.0, 2.0)
    assert got.shape == ref.shape and got.dtype == ref.dtype
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("shape,dt,gsig,tsig,bc", [
    ((31, 37), np.float32, 1.0, 2.0, "mirror"),
    ((40, 33), np.uint16, 1.5, 4.0, "periodic"),
    ((1, 25, 27), np.float32, 1.0, 3.0, "add zeros"),
    ((12, 1, 19), np.uint8, 1.0, 2.0, "zero order"),
    ((14, 15, 16), np.float32, 1.0, 4.0, "mirror"),
    ((9, 10, 11), np.int32, 0.9, 1.5, "asym mirror"),
    ((9, 10, 11), np.float64, 1.2, 2.0, "first order"),
    ((21, 18, 17), np.int16, 1.0, 2.5, "third order"),
    ((50,), np.float32, 1.0, 2.0, "antisym reflect"),
])
def test_forward_matches_oracle(cuda, shape, dt, gsig, tsig, bc):
    rng = np.random.default_rng(zlib.crc32(repr((shape, bc)).encode()))
    x = (rng.random(shape) * 200).astype(dt)
    ref = oracle.structure_tensor(x, gsig, tsig, bc, 3.0)
    got = st_gpu(x, gsig, tsig, bc)
    assert got.shape == ref.shape and got.dtype == ref.dtype
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


def test_per_axis_sigmas_and_zero_sigma_axis(cuda):
    import diplib_b200 as dip
    rng = np.random.default_rng(5)
    x = rng.random((11, 13, 15)).astype(np.float32)
    got = dip.StructureTensor(x, None, [1.0, 0.0, 1.5], [2.0, 3.0, 1.0], "gaussFIR", ["mirror", "periodic", "mirror"])
    ref = oracle.structure_tensor(x, [1.0, 0.0, 1.5], [2.0, 3.0, 1.0], ["mirror", "periodic", "mirror"], 3.0)
    assert got.shape == (3, 11, 13, 15) == ref.shape
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


def test_interleaved_output_layout_through_the_c_abi(cuda):
    """DIPlib's own layout: tensor stride 1, pixel strides multiplied by the component count."""
    import diplib_b200 as dip
    from diplib_b200 import _abi
    rng = np.random.default_rng(9)
    x = rng.random((8, 9, 10)).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    out = torch.full((8, 9, 10, 6), float("nan"), dtype=torch.float32, device="cuda")
    din = dip.image_desc(xt)
    dout = _abi.ImageDesc()
    dout.data = out.data_ptr()
    dout.dtype = _abi.SFLOAT
    dout.ndims = 4
    for i, (s, st) in enumerate([(10, 6), (9, 60), (8, 540), (6, 1)]):
        dout.sizes[i] = s
        dout.strides[i] = st
    three = (ctypes.c_double * 3)
    st = _abi.lib().dipcu_structure_tensor(ctypes.byref(din), ctypes.byref(dout), three(1.0, 1.0, 1.0),
                                           three(2.0, 2.0, 2.0), (ctypes.c_int32 * 3)(0, 0, 0), 3.0, None)
    assert st == 0, _abi.last_error()
    torch.cuda.synchronize()
    ref = oracle.structure_tensor(x, 1.0, 2.0, "mirror", 3.0)
    got = np.moveaxis(out.cpu().numpy(), -1, 0)
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


def test_errors(cuda):
    import diplib_b200 as dip
    with pytest.raises(dip.ParameterError):
        dip.StructureTensor(np.zeros((1, 1), np.float32), None, 1.0, 2.0, "gaussFIR")
    with pytest.raises(dip.ParameterError):
        dip.StructureTensor(np.zeros((8, 8), np.float32), None, 1.0, 2.0, "bogus")
    with pytest.raises(NotImplementedError):
        dip.StructureTensor(np.zeros((8, 8), np.float32), None, 1.0, 2.0, "finitediff")
    with pytest.raises(NotImplementedError):
        dip.StructureTensor(np.zeros((8, 8), np.float32), np.ones((8, 8), bool), 1.0, 2.0)
    with pytest.raises(dip.ParameterError):
        dip.StructureTensor(np.zeros((8, 8), np.float32), None, 1.0, 2.0, "gaussFIR", "no such bc")


def test_full_size_volume_forward(cuda):
    x = smoothed_noise(101, (192, 192, 192))
    ref = oracle.structure_tensor(x, 1.0, 4.0, "mirror", 3.0)
    got = st_gpu(x, 1.0, 4.0)
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


# ---- backward ------------------------------------------------------------------------------------

def st_backward_gpu(x: np.ndarray, w: np.ndarray, gsig, tsig, bc) -> np.ndarray:
    from diplib_b200 import torch_ops
    xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    wt = torch.from_numpy(np.ascontiguousarray(w)).cuda()
    g = torch_ops.structure_tensor_backward(wt, xt, gsig, tsig, bc, 3.0)
    return g.cpu().numpy()


@pytest.mark.parametrize("shape,gsig,tsig,bc", [
    ((9, 10, 11), 1.0, 2.0, "mirror"),
    ((9, 10, 11), 1.0, 4.0, "mirror"),
    ((12, 13), 1.3, 2.0, "periodic"),
    ((1, 10, 12), 1.0, 2.0, "zero order"),
    ((8, 9, 7), 0.9, 1.5, "asym mirror"),
    ((10, 11), 1.0, 2.0, "second order"),
])
def test_backward_vs_fp64_finite_differences(cuda, shape, gsig, tsig, bc):
    rng = np.random.default_rng(len(shape) * 1000 + int(gsig * 10) + int(tsig * 100))
    x = rng.standard_normal(shape)
    ncomp = oracle.structure_tensor(x, gsig, tsig, bc, 3.0).shape[0]
    w = rng.standard_normal((ncomp,) + shape)
    gx = st_backward_gpu(x, w, gsig, tsig, bc)
    h = 1e-2   # T is quadratic in x: the central difference is exact up to rounding
    flat = rng.choice(x.size, 40, replace=False)
    fd, got = [], []
    for f in flat:
        idx = np.unravel_index(f, shape)
        xp, xm = x.copy(), x.copy()
        xp[idx] += h
        xm[idx] -= h
        lp = float((w * oracle.structure_tensor(xp, gsig, tsig, bc, 3.0)).sum())
        lm = float((w * oracle.structure_tensor(xm, gsig, tsig, bc, 3.0)).sum())
        fd.append((lp - lm) / (2 * h))
        got.append(gx[idx])
    fd, got = np.array(fd), np.array(got)
    assert np.abs(got - fd).max() <= 1e-8 * max(1.0, np.abs(fd).max()), np.abs(got - fd).max()


def test_backward_float32_matches_float64(cuda):
    rng = np.random.default_rng(17)
    x = smoothed_noise(17, (24, 26, 28)).astype(np.float64)
    w = rng.standard_normal((6, 24, 26, 28))
    g64 = st_backward_gpu(x, w, 1.0, 4.0, "mirror")
    g32 = st_backward_gpu(x.astype(np.float32), w.astype(np.float32), 1.0, 4.0, "mirror")
    assert np.abs(g32 - g64).max() <= 1e-5 * np.abs(g64).max()


def test_full_size_backward_homogeneity_identity(cuda):
    """<dL/dx, x> = 2 L for the degree-2 homogeneous T, on one 192^3 volume of the workload."""
    from diplib_b200 import torch_ops
    x = torch.from_numpy(smoothed_noise(103, (192, 192, 192))).cuda()
    g = torch.Generator(device="cuda").manual_seed(104)
    w = torch.randn((6, 192, 192, 192), generator=g, device="cuda")
    t = torch_ops.structure_tensor(x, 1.0, 4.0, "mirror", 3.0)
    loss = (w.double() * t.double()).sum()
    gx = torch_ops.structure_tensor_backward(w, x, 1.0, 4.0, "mirror", 3.0)
    lhs = (gx.double() * x.double()).sum()
    assert abs(float(lhs) - 2 * float(loss)) <= 1e-4 * float((w.double().abs() * t.double().abs()).sum())


def test_autograd_gradcheck(cuda):
    from diplib_b200 import torch_ops
    g = torch.Generator().manual_seed(23)
    x = torch.randn((5, 6, 7), generator=g, dtype=torch.float64).cuda().requires_grad_()
    assert torch.autograd.gradcheck(lambda xx: torch_ops.structure_tensor(xx, 1.0, 2.0, "mirror", 3.0), (x,),
                                    eps=1e-6, atol=1e-7, rtol=1e-5)


def test_autograd_batch_loss(cuda):
    """The workload's loss over a batch of volumes: one backward call per volume."""
    from diplib_b200 import torch_ops
    rng = np.random.default_rng(29)
    xs = [torch.from_numpy(rng.standard_normal((10, 11, 12)).astype(np.float32)).cuda().requires_grad_()
          for _ in range(3)]
    ws = [torch.from_numpy(rng.standard_normal((6, 10, 11, 12)).astype(np.float32)).cuda() for _ in range(3)]
    loss = sum((w * torch_ops.structure_tensor(x, 1.0, 4.0, "mirror")).sum() for x, w in zip(xs, ws))
    loss.backward()
    for x, w in zip(xs, ws):
        ref = st_backward_gpu(x.detach().cpu().numpy().astype(np.float64), w.cpu().numpy().astype(np.float64),
                              1.0, 4.0, "mirror")
        assert np.abs(x.grad.cpu().numpy() - ref).max() <= 1e-5 * np.abs(ref).max()
