"""The 2D warp-per-tile kernel (half-width buckets 4, 6, 9, 12 with runtime taps and symmetry)
against the oracle: every sigma / derivative-order combination of the batched workload's set that
fits a bucket, tiles straddling the image edges, every x-y boundary condition it handles plus the
ones it hands back to the previous kernels, uint16 and float input, a batch axis, a cropped view
and an output with an odd row stride."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from tests.test_gauss_gpu import assert_close, dip, to_dev

pytestmark = pytest.mark.gpu

COMBOS = [(s, ox, oy) for s in (0.8, 1.0, 2.0, 3.0) for ox in range(3) for oy in range(3)] + [(4.0, 0, 0), (3.0, 2, 0)]


@pytest.mark.parametrize("sig,ox,oy", COMBOS)
def test_sigma_order_combinations(cuda, sig, ox, oy):
    rng = np.random.default_rng(int(sig * 100) + 10 * ox + oy)
    x = rng.random((77, 131), dtype=np.float32)
    ref = oracle.gauss_fir(x, [sig, sig], [ox, oy], ["mirror"], 3.0)
    got = dip().GaussFIR(x, [sig, sig], [ox, oy], ["mirror"], 3.0)
    assert_close(got, ref, x, f"{sig} {ox} {oy}")


@pytest.mark.parametrize("shape,dt,sig,ords,bcs", [
    ((64, 64), np.float32, (2.0, 2.0), (0, 0), ("mirror", "mirror")),
    ((1024, 1024), np.float32, (2.0, 2.0), (0, 0), ("mirror", "mirror")),
    ((300, 257), np.float32, (3.0, 3.0), (1, 0), ("zero order", "add zeros")),
    ((129, 95), np.float32, (1.5, 2.5), (0, 1), ("asym mirror", "mirror")),
    ((200, 201), np.uint16, (2.0, 1.0), (2, 1), ("mirror", "zero order")),
    ((33, 47), np.uint16, (3.0, 3.0), (0, 0), ("add zeros", "add zeros")),
    ((40, 50), np.float32, (1.0, 1.0), (0, 0), ("periodic", "periodic")),          # previous kernel
    ((10, 200), np.float32, (3.0, 3.0), (0, 0), ("mirror", "mirror")),              # ny <= bucket: previous kernel
])
def test_edges_and_boundary_conditions(cuda, shape, dt, sig, ords, bcs):
    rng = np.random.default_rng(shape[0] * 1000 + shape[1])
    x = rng.integers(0, 4096, size=shape, dtype=np.uint16) if dt == np.uint16 else rng.random(shape, dtype=np.float32)
    ref = oracle.gauss_fir(x, list(sig), list(ords), list(bcs), 3.0)
    got = dip().GaussFIR(x, list(sig), list(ords), list(bcs), 3.0)
    assert_close(got, ref, x, str((shape, sig, ords, bcs)))


def test_batch_axis_view_and_odd_output_stride(cuda):
    rng = np.random.default_rng(3)
    x = rng.random((5, 70, 90), dtype=np.float32)       # 2D filter with an unfiltered batch axis
    ref = oracle.gauss_fir(x, [2.0, 2.0, 0.0], [1, 0, 0], ["mirror"], 3.0)
    got = dip().GaussFIR(x, [2.0, 2.0, 0.0], [1, 0, 0], ["mirror"], 3.0)
    assert_close(got, ref, x, "batch")
    big = rng.random((100, 128), dtype=np.float32)
    view = to_dev(big)[7:90, 4:120]
    ref = oracle.gauss_fir(np.ascontiguousarray(big[7:90, 4:120]), [2.0, 2.0], [0, 0], ["mirror"], 3.0)
    got = dip().GaussFIR(view, [2.0, 2.0], [0, 0], ["mirror"], 3.0).cpu().numpy()
    assert_close(got, ref, big, "view")
    out_full = torch.full((60, 81), float("nan"), device="cuda")
    out = out_full[:, :80]
    x2 = rng.random((60, 80), dtype=np.float32)
    dip().GaussFIR(to_dev(x2), [2.0, 2.0], [0, 0], ["mirror"], 3.0, out=out)
    assert_close(out.cpu().numpy(), oracle.gauss_fir(x2, [2.0, 2.0], [0, 0], ["mirror"], 3.0), x2, "odd stride")
    assert torch.isnan(out_full[:, 80]).all()
