"""The batched workload exactly as bench.py times it: the 512 uneven 2D images of
``bench.make_batch_params(seed=0)`` with the bench's inputs (torch.rand, generator seed 20 on the
device), one plan with graph capture and autotuning.  Every image of the first run (the capture)
and of a graph replay is checked against the oracle (the restated dip::GaussFIR per image,
src/linear/gauss.cpp:238-286 in DIPlib) at <= 1e-5 of the input range; the error against the FP64
oracle is reported for a subset.  Run with ``-s`` to print the errors."""
from __future__ import annotations

import concurrent.futures
import os

import numpy as np
import pytest
import torch

import bench
import oracle

pytestmark = pytest.mark.gpu


def _oracle_all(imgs, params, dtype):
    # ctypes releases the GIL during the oracle's C calls, so threads run the images in parallel.
    def one(i):
        s, o, bc = params[i]
        return oracle.gauss_fir(imgs[i].astype(dtype), [s, s], o, [bc], 3.0)
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 8) as ex:
        return list(ex.map(one, range(len(imgs))))


def test_bench_batch_plan_matches_oracle(cuda):
    from diplib_b200.batch import BatchPlan, device_status
    device_status(clear=True)
    shapes, params = bench.make_batch_params(seed=0)
    assert len(shapes) == 512
    gen = torch.Generator(device=cuda).manual_seed(20)
    ins = [torch.rand(s, generator=gen, device=cuda) for s in shapes]
    outs = [torch.full(s, float("nan"), device=cuda) for s in shapes]
    plan = BatchPlan(ins, outs, [p[0] for p in params], [p[1] for p in params], [p[2] for p in params],
                     graph=True, autotune=True)
    imgs = [t.cpu().numpy() for t in ins]
    refs = _oracle_all(imgs, params, np.float32)
    try:
        for run in ("first run", "graph replay"):
            for o in outs:
                o.fill_(float("nan"))
            plan.run()
            torch.cuda.synchronize()
            assert device_status(clear=True) == 0
            worst = 0.0
            for i, (a, r) in enumerate(zip(imgs, refs)):
                got = outs[i].cpu().numpy()
                err = float(np.abs(got - r).max())     # NaN (an unwritten pixel) fails the bar too
                tol = 1e-5 * float(a.max() - a.min())
                assert err <= tol, (run, i, a.shape, params[i], err)
                worst = max(worst, err)
            print(f"\n[batch 512, {run}] max abs error against the float32 oracle {worst:.3e}")
        # FP64 oracle on every 16th image
        sub = list(range(0, 512, 16))
        r64 = _oracle_all([imgs[i] for i in sub], [params[i] for i in sub], np.float64)
        worst64 = max(float(np.abs(outs[i].cpu().numpy() - r).max()) for i, r in zip(sub, r64))
        print(f"[batch 512] max abs error against the FP64 oracle over {len(sub)} images {worst64:.3e}")
        assert worst64 <= 1e-5
    finally:
        plan.close()
