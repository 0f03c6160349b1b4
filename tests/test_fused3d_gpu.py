"""The 3D fused tile kernels against the oracle on the shapes that stress their geometry: tile
columns that straddle the image edge in x and y (partial tiles, the tile origin offset), z chunks
split across CTAs, volumes thinner than the z kernel (multi-bounce z mirror), every x-y boundary
condition the warp-specialised kernel handles plus the ones it hands back to the previous kernel,
a batch axis, strided inputs and unaligned output strides."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from tests.test_gauss_gpu import assert_close, dip, to_dev

pytestmark = pytest.mark.gpu

# (shape (z, y, x), dtype, sigmas (x, y, z), orders (x, y, z), bcs (x, y, z))
CASES = [
    ((41, 37, 103), np.uint16, (1.5, 1.5, 3.0), (0, 0, 0), ("mirror",) * 3),
    ((41, 37, 103), np.uint16, (1.5, 1.5, 3.0), (1, 0, 0), ("mirror",) * 3),
    ((30, 19, 49), np.uint16, (1.5, 1.5, 3.0), (1, 0, 0), ("zero order",) * 3),
    ((25, 33, 130), np.float32, (1.5, 1.5, 3.0), (0, 0, 0), ("add zeros",) * 3),
    ((5, 23, 61), np.uint16, (1.5, 1.5, 3.0), (0, 0, 0), ("mirror",) * 3),         # nz < HZ
    ((64, 16, 48), np.uint16, (1.5, 1.5, 3.0), (0, 0, 0), ("mirror", "mirror", "periodic")),
    ((29, 21, 60), np.float32, (1.0, 1.0, 1.0), (1, 0, 0), ("asym mirror",) * 3),
    ((29, 21, 60), np.float32, (1.0, 1.0, 1.0), (0, 1, 0), ("asym mirror",) * 3),
    ((29, 21, 60), np.float32, (1.0, 1.0, 1.0), (0, 0, 1), ("asym mirror",) * 3),
    ((29, 21, 60), np.float32, (1.0, 1.0, 1.0), (0, 0, 0), ("mirror", "zero order", "asym periodic")),
    ((17, 9, 70), np.float32, (1.0, 1.0, 1.0), (0, 0, 0), ("periodic",) * 3),       # previous kernel
    ((40, 50, 120), np.float32, (4.0, 4.0, 4.0), (0, 0, 0), ("mirror",) * 3),
    ((12, 5, 7), np.uint16, (1.5, 1.5, 3.0), (0, 0, 0), ("mirror",) * 3),           # n <= H in y: previous kernel
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-{np.dtype(c[1]).name}-{c[3]}-{c[4][0]}" for c in CASES])
def test_3d_kernels_against_oracle(cuda, case):
    shape, dt, sig, ords, bcs = case
    rng = np.random.default_rng(abs(hash(shape)) % 2**31)
    if dt == np.uint16:
        x = rng.integers(0, 4096, size=shape, dtype=np.uint16)
    else:
        x = rng.random(shape, dtype=np.float32)
    ref = oracle.gauss_fir(x, list(sig), list(ords), list(bcs), 3.0)
    got = dip().GaussFIR(x, list(sig), list(ords), list(bcs), 3.0)
    assert_close(got, ref, x, str(case))


def test_batch_axis_and_strided_input(cuda):
    rng = np.random.default_rng(7)
    # 4D with an unfiltered batch axis (sigma 0 on the 4th DIPlib axis).
    x = rng.integers(0, 4096, size=(3, 20, 30, 100), dtype=np.uint16)
    sig, ords = [1.5, 1.5, 3.0, 0.0], [0, 0, 0, 0]
    ref = oracle.gauss_fir(x, sig, ords, ["mirror"], 3.0)
    got = dip().GaussFIR(x, sig, ords, ["mirror"], 3.0)
    assert_close(got, ref, x, "batch")
    # A cropped view: row stride 128 samples, x size 100.
    big = rng.integers(0, 4096, size=(24, 40, 128), dtype=np.uint16)
    view = to_dev(big)[:, 3:37, 5:105]
    ref = oracle.gauss_fir(np.ascontiguousarray(big[:, 3:37, 5:105]), [1.5, 1.5, 3.0], [0, 0, 0], ["mirror"], 3.0)
    got = dip().GaussFIR(view, [1.5, 1.5, 3.0], [0, 0, 0], ["mirror"], 3.0).cpu().numpy()
    assert_close(got, ref, big, "view")


def test_unaligned_output_strides(cuda):
    rng = np.random.default_rng(11)
    x = rng.random((20, 30, 64), dtype=np.float32)
    ref = oracle.gauss_fir(x, [1.5, 1.5, 3.0], [0, 0, 0], ["mirror"], 3.0)
    out_full = torch.full((20, 30, 65), float("nan"), device="cuda")
    out = out_full[:, :, :64]                      # row stride 65: no 8-byte pair stores
    dip().GaussFIR(to_dev(x), [1.5, 1.5, 3.0], [0, 0, 0], ["mirror"], 3.0, out=out)
    assert_close(out.cpu().numpy(), ref, x, "odd stride")
    assert torch.isnan(out_full[:, :, 64]).all()
