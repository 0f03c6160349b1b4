"""The adjoint of the Gaussian FIR (dipcu_gauss_fir_backward) and the torch autograd wrapper.

Checks, on the configuration of the differentiable-Gaussian benchmark (sigma 3, orders (0,0),
(1,0), (0,1), (2,0), "mirror") and on every boundary condition:
  * against FP64 central finite differences (step 1e-3) on a seeded 64x64 crop, for the input
    gradient and for the sigma gradient (kernel length held fixed, as the analytic derivative is);
  * against a reference gradient built from dip::Gauss calls: per axis, in reverse pass order, a
    dip::Gauss with "add zeros" of the zero-padded upstream gradient (negated for odd orders, i.e.
    the correlation with the flipped kernel) followed by the transpose of the boundary extension
    (assembled from dip's ExpandBuffer applied to unit vectors);
  * torch.autograd.gradcheck in float64.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import oracle
from tests.conftest import HOSTLOGIC

pytestmark = pytest.mark.gpu

ORDERS4 = [(0, 0), (1, 0), (0, 1), (2, 0)]


def dip():
    import diplib_b200
    return diplib_b200


def tops():
    from diplib_b200 import torch_ops
    return torch_ops


def ext_matrix(n: int, h: int, bc: str) -> np.ndarray:
    """(n + 2h) x n matrix of the boundary extension (its linear part), from ExpandBuffer."""
    base = oracle.expand_buffer(np.zeros(n), h, h, bc)
    cols = []
    for i in range(n):
        e = np.zeros(n)
        e[i] = 1.0
        cols.append(oracle.expand_buffer(e, h, h, bc) - base)
    return np.stack(cols, axis=1)


def ref_input_grad(gy: np.ndarray, sig, ords, bcs, trunc=3.0, use_ref=False):
    """E^T C^T gy per axis in reverse pass order, built from dip::Gauss calls (float64)."""
    nd = gy.ndim
    gauss = oracle.ref_gauss if use_ref else oracle.gauss_fir
    g = gy.astype(np.float64)
    dims = [d for d in range(nd) if sig[d] > 0 and gy.shape[nd - 1 - d] > 1]
    for d in reversed(dims):          # forward order is x first (smallest stride)
        ax = nd - 1 - d
        h = oracle.half_gaussian(sig[d], ords[d], trunc, True).size - 1
        pad = [(0, 0)] * nd
        pad[ax] = (h, h)
        gp = np.pad(g, pad)
        s1 = [0.0] * nd
        s1[d] = sig[d]
        o1 = [0] * nd
        o1[d] = ords[d]
        z = gauss(gp, s1, o1, ["add zeros"], trunc)
        if ords[d] % 2:
            z = -z
        E = ext_matrix(g.shape[ax], h, bcs[d])
        g = np.moveaxis(np.tensordot(z, E, axes=([ax], [0])), -1, ax)
    return g


def gpu_backward(x: np.ndarray, gy: np.ndarray, sig, ords, bcs, trunc=3.0, need_sigma=True):
    xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    gt = torch.from_numpy(np.ascontiguousarray(gy)).cuda()
    gx, gs = tops().gauss_backward(gt, xt, sig, ords, bcs, trunc, True, need_sigma)
    torch.cuda.synchronize()
    return gx.cpu().numpy(), (gs.cpu().numpy() if gs is not None else None)


@pytest.mark.parametrize("ords", ORDERS4)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_input_gradient_vs_fp64_finite_differences(cuda, ords, dtype):
    rng = np.random.default_rng(41)
    x = rng.random((64, 64))
    gy = rng.standard_normal((64, 64))
    sig = [3.0, 3.0]
    bcs = ["mirror", "mirror"]
    gx, _ = gpu_backward(x.astype(dtype), gy.astype(dtype), sig, list(ords), bcs, need_sigma=False)
    h = 1e-3
    idx = list(zip(rng.integers(0, 64, 300), rng.integers(0, 64, 300)))
    idx += [(r, c) for r in (0, 1, 2, 61, 62, 63) for c in range(0, 64, 3)]
    fd = []
    for r, c in idx:
        xp, xm = x.copy(), x.copy()
        xp[r, c] += h
        xm[r, c] -= h
        lp = float((gy * oracle.gauss_fir(xp, sig, list(ords), bcs)).sum())
        lm = float((gy * oracle.gauss_fir(xm, sig, list(ords), bcs)).sum())
        fd.append((lp - lm) / (2 * h))
    fd = np.array(fd)
    got = np.array([gx[r, c] for r, c in idx])
    tol = (1e-9 if dtype == np.float64 else 2e-5) * np.abs(fd).max() + 1e-9
    assert np.abs(got - fd).max() <= tol, np.abs(got - fd).max()


def _fixed_length_loss(x, gy, sig, ords, bcs, trunc, axis, s_axis):
    """FP64 forward with the kernel of `axis` built for sigma `s_axis` at the length sigma gives."""
    l = ctypes.CDLL(HOSTLOGIC)
    l.hl_half_gaussian_length.restype = ctypes.c_int64
    l.hl_half_gaussian_length.argtypes = [ctypes.c_double, ctypes.c_uint32, ctypes.c_double, ctypes.c_int]
    l.hl_make_half_gaussian.argtypes = [ctypes.c_double, ctypes.c_uint32, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    taps = []
    for d in range(len(sig)):
        n = l.hl_half_gaussian_length(sig[d], ords[d], trunc, 1)
        w = np.zeros(n)
        l.hl_make_half_gaussian(s_axis if d == axis else sig[d], ords[d], n, w.ctypes.data, None)
        taps.append(w)
    y = oracle.separable_fir(x, taps, [o % 2 for o in ords], bcs)
    return float((gy * y).sum())


@pytest.mark.parametrize("ords", ORDERS4)
def test_sigma_gradient_vs_fp64_finite_differences(cuda, ords):
    rng = np.random.default_rng(43)
    x = rng.random((64, 64))
    gy = rng.standard_normal((64, 64))
    sig = [3.0, 3.0]
    bcs = ["mirror", "mirror"]
    _, gs = gpu_backward(x.astype(np.float32), gy.astype(np.float32), sig, list(ords), bcs)
    h = 1e-3
    for axis in range(2):
        fd = (_fixed_length_loss(x, gy, sig, list(ords), bcs, 3.0, axis, sig[axis] + h) -
              _fixed_length_loss(x, gy, sig, list(ords), bcs, 3.0, axis, sig[axis] - h)) / (2 * h)
        assert abs(gs[axis] - fd) <= 1e-4 * max(1.0, abs(fd)), (axis, gs[axis], fd)


@pytest.mark.parametrize("bc", ["mirror", "asym mirror", "periodic", "asym periodic", "add zeros", "zero order",
                                "first order", "second order", "third order", "antisym reflect", "add max"])
def test_input_gradient_vs_reference_built_gradient(cuda, bc):
    rng = np.random.default_rng(47)
    x = rng.random((23, 31))
    gy = rng.standard_normal((23, 31))
    for sig, ords in [([3.0, 3.0], [0, 0]), ([2.0, 1.5], [1, 2]), ([1.2, 4.0], [3, 1])]:
        gx, _ = gpu_backward(x, gy, sig, ords, [bc, bc], need_sigma=False)
        ref = ref_input_grad(gy, sig, ords, [bc, bc], use_ref=oracle.ref_available())
        assert np.abs(gx - ref).max() <= 1e-9 * np.abs(ref).max() + 1e-12, (bc, sig, ords)


def test_3d_and_multi_reflection_input_gradient(cuda):
    rng = np.random.default_rng(53)
    gy = rng.standard_normal((6, 9, 11))
    x = rng.random((6, 9, 11))
    for bc in ["mirror", "periodic", "zero order"]:
        sig, ords = [2.5, 1.0, 3.0], [0, 1, 2]
        gx, _ = gpu_backward(x, gy, sig, ords, [bc] * 3, need_sigma=False)
        ref = ref_input_grad(gy, sig, ords, [bc] * 3)
        assert np.abs(gx - ref).max() <= 1e-9 * np.abs(ref).max(), bc


def test_full_size_2048_input_gradient(cuda):
    rng = np.random.default_rng(59)
    x = rng.random((2048, 2048), dtype=np.float32)
    gy = rng.standard_normal((2048, 2048)).astype(np.float32)
    for ords in ORDERS4:
        gx, _ = gpu_backward(x, gy, [3.0, 3.0], list(ords), ["mirror", "mirror"], need_sigma=False)
        ref = ref_input_grad(gy.astype(np.float64), [3.0, 3.0], list(ords), ["mirror", "mirror"])
        assert np.abs(gx - ref).max() <= 1e-5 * np.abs(ref).max(), ords


def test_autograd_gradcheck(cuda):
    g = torch.Generator().manual_seed(61)
    x = torch.rand((12, 14), generator=g, dtype=torch.float64).cuda().requires_grad_()
    s = torch.tensor([1.3, 2.2], dtype=torch.float64).cuda().requires_grad_()
    for order in ([0, 0], [1, 0], [2, 1]):
        fn = lambda xx, ss: tops().gauss(xx, ss, order, ["mirror"], 3.0)  # noqa: E731
        assert torch.autograd.gradcheck(fn, (x, s), eps=1e-6, atol=1e-7, rtol=1e-5)
    # Scalar sigma: the gradient is the sum over axes.
    s1 = torch.tensor(1.7, dtype=torch.float64).cuda().requires_grad_()
    assert torch.autograd.gradcheck(lambda xx, ss: tops().gauss(xx, ss, [1, 0], ["periodic"], 3.0), (x, s1),
                                    eps=1e-6, atol=1e-7, rtol=1e-5)


@pytest.mark.parametrize("case", [
    ((48, 50), np.float32, [3.0, 3.0], [2, 1], "mirror"),
    ((3, 40, 52), np.float32, [2.0, 1.5, 0.0], [1, 0, 0], "asym mirror"),      # batch axis
    ((45, 60), np.uint16, [1.5, 2.5], [0, 1], "zero order"),
    ((33, 70), np.float32, [4.0, 1.0], [0, 2], "add zeros"),
])
def test_fused_adjoint_matches_pass_by_pass_adjoint(cuda, case, monkeypatch):
    """The one-kernel 2D backward against the pass-by-pass adjoint (line passes + halo folds) on
    the same inputs: input gradient, sigma gradients, a batch axis, integer input."""
    shape, dt, sig, ords, bc = case
    rng = np.random.default_rng(sum(shape))
    x = (rng.random(shape) * 1000).astype(dt) if dt == np.uint16 else rng.random(shape).astype(dt)
    gy = rng.standard_normal(shape).astype(np.float32)
    xt = torch.from_numpy(x.view(np.int16) if dt == np.uint16 else x).cuda()
    if dt == np.uint16:
        xt = xt.view(torch.uint16)
    gt = torch.from_numpy(gy).cuda()
    bcs = [bc] * len(shape)
    gx1, gs1 = tops().gauss_backward(gt, xt, sig, ords, bcs, 3.0, True, True)
    gx_only, _ = tops().gauss_backward(gt, xt, sig, ords, bcs, 3.0, True, False)
    _, gs_only = tops().gauss_backward(gt, xt, sig, ords, bcs, 3.0, False, True)
    torch.cuda.synchronize()
    monkeypatch.setenv("DIPCU_NO_WS", "1")
    gx2, gs2 = tops().gauss_backward(gt, xt, sig, ords, bcs, 3.0, True, True)
    torch.cuda.synchronize()
    g1, g2 = gx1.cpu().numpy(), gx2.cpu().numpy()
    assert np.abs(g1 - g2).max() <= 1e-5 * np.abs(g2).max()
    assert np.abs(gx_only.cpu().numpy() - g1).max() <= 1e-6 * np.abs(g1).max()
    s1, s2 = gs1.cpu().numpy(), gs2.cpu().numpy()
    assert np.allclose(s1, s2, rtol=1e-4, atol=1e-4 * np.abs(s2).max()), (s1, s2)
    assert np.allclose(gs_only.cpu().numpy(), s1, rtol=1e-6, atol=1e-9)
