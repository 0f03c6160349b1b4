"""The row-march 2D kernel (march2d.cuh: strips of 128 columns, runtime taps up to half-width 32
on each axis) against the oracle: every sigma / derivative-order / boundary-condition combination
of the batched workload, images narrower than a strip and shorter than the filter (boundary
extensions that bounce more than once), row runs split over several items, uint16 input, every
index-mapping boundary condition and "add zeros" on either axis, and a batch axis."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from tests.test_gauss_gpu import assert_close, dip

pytestmark = pytest.mark.gpu

SIGMAS = (0.8, 1.0, 2.0, 4.0, 8.0)
BCS = ("mirror", "periodic", "add zeros")


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("sig", SIGMAS)
def test_batch_combinations(cuda, sig, bc):
    rng = np.random.default_rng(int(sig * 10) + 7 * BCS.index(bc))
    x = rng.random((150, 300), dtype=np.float32)
    for ox in range(3):
        for oy in range(3):
            ref = oracle.gauss_fir(x, [sig, sig], [ox, oy], [bc], 3.0)
            got = dip().GaussFIR(x, [sig, sig], [ox, oy], [bc], 3.0)
            assert_close(got, ref, x, f"{sig} {ox} {oy} {bc}")


@pytest.mark.parametrize("shape,dt,sig,ords,bcs", [
    ((2000, 700), np.float32, (4.0, 4.0), (1, 2), ("periodic", "periodic")),        # many row runs
    ((3000, 130), np.float32, (8.0, 2.0), (2, 0), ("mirror", "add zeros")),
    ((500, 40), np.float32, (8.0, 8.0), (0, 1), ("mirror", "mirror")),              # narrower than a strip
    ((10, 300), np.float32, (4.0, 4.0), (0, 0), ("mirror", "mirror")),              # rows bounce several times
    ((9, 20), np.float32, (8.0, 8.0), (2, 2), ("periodic", "mirror")),              # both axes bounce
    ((257, 385), np.float32, (3.0, 2.0), (1, 1), ("asym mirror", "asym periodic")),
    ((131, 259), np.float32, (2.0, 5.0), (0, 3), ("zero order", "asym mirror")),
    ((400, 333), np.uint16, (2.0, 6.0), (1, 0), ("mirror", "periodic")),
    ((64, 4096), np.uint16, (7.5, 1.0), (0, 2), ("add zeros", "zero order")),
])
def test_shapes_types_and_boundaries(cuda, shape, dt, sig, ords, bcs):
    rng = np.random.default_rng(shape[0] + 7 * shape[1])
    x = rng.integers(0, 4096, size=shape, dtype=np.uint16) if dt == np.uint16 else rng.random(shape, dtype=np.float32)
    ref = oracle.gauss_fir(x, list(sig), list(ords), list(bcs), 3.0)
    got = dip().GaussFIR(x, list(sig), list(ords), list(bcs), 3.0)
    assert_close(got, ref, x, str((shape, sig, ords, bcs)))


def test_batch_axis(cuda):
    rng = np.random.default_rng(4)
    x = rng.random((3, 90, 260), dtype=np.float32)
    ref = oracle.gauss_fir(x, [6.0, 4.0, 0.0], [2, 1, 0], ["periodic", "mirror", "mirror"], 3.0)
    got = dip().GaussFIR(x, [6.0, 4.0, 0.0], [2, 1, 0], ["periodic", "mirror", "mirror"], 3.0)
    assert_close(got, ref, x, "batch axis")


@pytest.mark.parametrize("sig,ords,bcs", [((8.0, 8.0), (0, 2), ("mirror", "periodic")),
                                          ((4.0, 6.0), (1, 0), ("add zeros", "asym mirror")),
                                          ((2.0, 2.0), (0, 0), ("periodic", "mirror"))])
def test_rows_tma_cannot_address(cuda, sig, ords, bcs):
    """Views whose row stride is not a multiple of 16 bytes: the stages are filled by per-thread
    asynchronous copies instead of TMA."""
    import torch
    from tests.test_gauss_gpu import to_dev
    rng = np.random.default_rng(21)
    big = rng.random((310, 333), dtype=np.float32)
    view = to_dev(big)[3:300, 1:330]                      # row stride 333 floats, origin 4-byte aligned
    x = np.ascontiguousarray(big[3:300, 1:330])
    ref = oracle.gauss_fir(x, list(sig), list(ords), list(bcs), 3.0)
    out = torch.empty((297, 329), device="cuda")
    dip().GaussFIR(view, list(sig), list(ords), list(bcs), 3.0, out=out)
    assert_close(out.cpu().numpy(), ref, x, str((sig, ords, bcs)))
