"""Error of the GPU path against the FP64 oracle (the restated dip::Gauss run on float64 input),
for each benchmark configuration at its full size, plus the bar: max abs error <= 1e-5 times the
input range (for derivatives and the structure tensor, times the reference's magnitude).
Run with ``-s`` to print the measured errors."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def report(name, err, scale):
    print(f"\n[fp64 error] {name}: max abs err {err:.3e} = {err / scale:.3e} x scale ({scale:.4g})")
    assert err <= 1e-5 * scale, (name, err, scale)


def test_plain_2d_1024(cuda):
    import diplib_b200 as dip
    x = np.random.default_rng(0).random((1024, 1024), dtype=np.float32)
    got = dip.GaussFIR(x, [2.0, 2.0], [0, 0], ["mirror"], 3.0)
    ref = oracle.gauss_fir(x.astype(np.float64), [2.0, 2.0], [0, 0], ["mirror"], 3.0)
    report("2D 1024^2 sfloat sigma 2", float(np.abs(got - ref).max()), float(x.max() - x.min()))


@pytest.mark.parametrize("order", [[0, 0, 0], [1, 0, 0]])
def test_3d_256_uint16(cuda, order):
    import diplib_b200 as dip
    x = np.random.default_rng(0).integers(0, 4096, size=(256, 256, 256), dtype=np.uint16)
    got = dip.GaussFIR(x, [1.5, 1.5, 3.0], order, ["mirror"], 3.0)
    ref = oracle.gauss_fir(x.astype(np.float64), [1.5, 1.5, 3.0], order, ["mirror"], 3.0)
    report(f"3D 256^3 uint16 order {order}", float(np.abs(got - ref).max()), 4095.0)


def test_batched_sample(cuda):
    from diplib_b200.batch import BatchPlan
    rng = np.random.default_rng(5)
    imgs, params = [], []
    for _ in range(24):
        h, w = (int(v) for v in rng.integers(64, 2049, 2))
        imgs.append(rng.random((h, w), dtype=np.float32))
        params.append((float(rng.choice([0.8, 1.0, 2.0, 4.0, 8.0])), [int(rng.integers(0, 3)), int(rng.integers(0, 3))],
                       str(rng.choice(["mirror", "periodic", "add zeros"]))))
    ins = [torch.from_numpy(a).cuda() for a in imgs]
    outs = [torch.empty_like(t) for t in ins]
    plan = BatchPlan(ins, outs, [p[0] for p in params], [p[1] for p in params], [p[2] for p in params])
    plan.run()
    torch.cuda.synchronize()
    worst = 0.0
    for a, o, (s, ords, bc) in zip(imgs, outs, params):
        ref = oracle.gauss_fir(a.astype(np.float64), [s, s], ords, [bc], 3.0)
        worst = max(worst, float(np.abs(o.cpu().numpy() - ref).max()))
    plan.close()
    report("batched, 24 images of the uneven batch", worst, 1.0)


@pytest.mark.parametrize("order", [[0, 0], [1, 0], [0, 1], [2, 0]])
def test_differentiable_2d_2048(cuda, order):
    import diplib_b200 as dip
    from diplib_b200 import torch_ops
    from tests.test_backward_gpu import ref_input_grad
    rng = np.random.default_rng(11)
    x = rng.random((2048, 2048), dtype=np.float32)
    gy = rng.standard_normal((2048, 2048)).astype(np.float32)
    got = dip.GaussFIR(x, [3.0, 3.0], order, ["mirror"], 3.0)
    ref = oracle.gauss_fir(x.astype(np.float64), [3.0, 3.0], order, ["mirror"], 3.0)
    report(f"2D 2048^2 forward order {order}", float(np.abs(got - ref).max()), 1.0)
    gx, _ = torch_ops.gauss_backward(torch.from_numpy(gy).cuda(), torch.from_numpy(x).cuda(), [3.0, 3.0], order,
                                     ["mirror"], 3.0, True, False)
    rg = ref_input_grad(gy.astype(np.float64), [3.0, 3.0], order, ["mirror", "mirror"])
    report(f"2D 2048^2 input gradient order {order}", float(np.abs(gx.cpu().numpy() - rg).max()), float(np.abs(rg).max()))


def test_structure_tensor_192(cuda):
    import diplib_b200 as dip
    from tests.test_structure_tensor_gpu import smoothed_noise
    x = smoothed_noise(101, (192, 192, 192))
    got = dip.StructureTensor(x, None, 1.0, 4.0, "gaussFIR", "mirror", 3.0)
    ref = oracle.structure_tensor(x.astype(np.float64), 1.0, 4.0, "mirror", 3.0)
    report("structure tensor 192^3", float(np.abs(got - ref).max()), float(np.abs(ref).max()))
