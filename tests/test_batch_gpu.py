"""The batched persistent launch (dipcu_batch_plan_*): every image of an uneven batch matches
the oracle, CUDA-graph replays and in-place sigma updates give the new filter, the autotuner
picks a valid tile shape, and a planted impossible work item is skipped and reported (the
kernel finishes; nothing on the GPU is made to fault or wait)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

SIGMAS = [0.8, 1.0, 2.0, 4.0, 8.0]
BCS = ["mirror", "periodic", "add zeros"]


def make_batch(n, seed, lo=20, hi=300):
    rng = np.random.default_rng(seed)
    imgs, params = [], []
    for _ in range(n):
        h, w = (int(v) for v in rng.integers(lo, hi + 1, 2))
        imgs.append(rng.random((h, w), dtype=np.float32))
        s = float(rng.choice(SIGMAS))
        params.append((s, [int(rng.integers(0, 3)), int(rng.integers(0, 3))], str(rng.choice(BCS))))
    return imgs, params


def run_plan(imgs, params, **kw):
    from diplib_b200.batch import BatchPlan
    ins = [torch.from_numpy(a).cuda() for a in imgs]
    outs = [torch.full_like(t, float("nan")) for t in ins]
    plan = BatchPlan(ins, outs, [p[0] for p in params], [p[1] for p in params], [p[2] for p in params], **kw)
    plan.run()
    torch.cuda.synchronize()
    return plan, ins, outs


def check_all(imgs, params, outs, sig_override=None):
    for i, (a, (s, o, bc)) in enumerate(zip(imgs, params)):
        sg = sig_override[i] if sig_override is not None else [s, s]
        ref = oracle.gauss_fir(a, sg, o, [bc], 3.0)
        got = outs[i].cpu().numpy()
        err = np.abs(got - ref).max()
        assert err <= 1e-5 * max(1.0, float(a.max() - a.min())), (i, a.shape, s, o, bc, err)


def test_batch_matches_oracle_with_graph_and_autotune(cuda):
    from diplib_b200.batch import device_status
    device_status(clear=True)
    imgs, params = make_batch(40, 1)
    plan, ins, outs = run_plan(imgs, params, graph=True, autotune=True)
    info = plan.info()
    assert info["tile"] in [(64, 32), (64, 16), (128, 32)] and info["items"] > 0
    check_all(imgs, params, outs)
    for o in outs:
        o.fill_(float("nan"))
    plan.run()                       # graph replay
    torch.cuda.synchronize()
    check_all(imgs, params, outs)
    assert device_status() == 0
    plan.close()


def test_batch_without_graph_and_small_images(cuda):
    imgs, params = make_batch(25, 2, lo=1, hi=40)
    plan, ins, outs = run_plan(imgs, params, graph=False, autotune=False)
    check_all(imgs, params, outs)
    plan.close()


def test_batch_sigma_table_update_between_replays(cuda):
    imgs, params = make_batch(12, 3)
    plan, ins, outs = run_plan(imgs, params, graph=True, autotune=False)
    tab = plan.sigma_table()
    # Shrink every sigma by 1e-4 (relative): no kernel length (ceil((3 + o/2) sigma)) changes for
    # this sigma set, so the captured graph stays valid and rebuilds the weights on the device.
    new = [[s * 0.9999, s * 0.9999] for s, _, _ in params]
    tab.copy_(torch.tensor([v for p in new for v in p], dtype=torch.float64, device=tab.device))
    plan.run()
    torch.cuda.synchronize()
    check_all(imgs, params, outs, sig_override=new)
    plan.close()


@pytest.mark.parametrize("flag", ["image", "tile"])
def test_batch_planted_invalid_item_is_skipped_and_reported(cuda, flag):
    from diplib_b200 import _abi
    from diplib_b200.batch import INJECT_INVALID_IMAGE, INJECT_INVALID_TILE, device_status
    device_status(clear=True)
    imgs, params = make_batch(10, 4)
    f = INJECT_INVALID_IMAGE if flag == "image" else INJECT_INVALID_TILE
    plan, ins, outs = run_plan(imgs, params, graph=True, autotune=False, flags=f)
    assert device_status(clear=True) == _abi.ERR_INVALID_ARG
    # Every other work item was filtered: at most one item's outputs are missing (an item is at most
    # one strip of 128 columns of one image).
    nan_count = sum(int(torch.isnan(o).sum()) for o in outs)
    assert 0 < nan_count <= 128 * max(a.shape[0] for a in imgs)
    plan.close()


def test_batch_tile_path_aligned_and_unaligned_rows(cuda):
    """Images the grouped tile path takes, with row strides that TMA can and cannot address
    (widths multiple of 4 and not), every bucket of half-widths, even and odd orders."""
    rng = np.random.default_rng(9)
    imgs, params = [], []
    for i, (w, s) in enumerate([(64, 0.8), (67, 1.0), (130, 2.0), (131, 2.0), (200, 3.0), (203, 3.0), (96, 4.0), (97, 4.0)]):
        imgs.append(rng.random((45 + 7 * i, w), dtype=np.float32))
        params.append((s, [i % 3, (i + 1) % 3] if s < 3 else [0, i % 2], ["mirror", "add zeros"][i % 2]))
    plan, ins, outs = run_plan(imgs, params, graph=False, autotune=False)
    check_all(imgs, params, outs)
    plan.close()


def test_batch_tile_path_periodic_edges(cuda):
    """Images the grouped tile path takes with "periodic" / "asym periodic" edges along one or
    both axes (their edge tiles gather the boxes with wrapped indices) beside "mirror" / "add
    zeros" along the other axis; widths multiple of 4 and not, one image narrower than a box."""
    rng = np.random.default_rng(11)
    cases = [(64, 0.8, ["periodic", "periodic"]), (67, 1.0, ["asym periodic", "mirror"]),
             (130, 2.0, ["mirror", "periodic"]), (131, 2.0, ["periodic", "add zeros"]),
             (200, 3.0, ["asym periodic", "asym periodic"]), (203, 1.0, ["add zeros", "asym periodic"]),
             (96, 4.0, ["periodic", "periodic"]), (26, 1.0, ["periodic", "asym periodic"])]
    imgs, params = [], []
    for i, (w, s, bc) in enumerate(cases):
        imgs.append(rng.random((45 + 7 * i, w), dtype=np.float32) - 0.5)
        params.append((s, [i % 3, (i + 1) % 3] if s < 3 else [0, i % 2], bc))
    plan, ins, outs = run_plan(imgs, params, graph=False, autotune=False)
    assert plan.info()["grouped_items"] > 0
    for i, (a, (s, o, bc)) in enumerate(zip(imgs, params)):
        ref = oracle.gauss_fir(a, [s, s], o, bc, 3.0)
        err = np.abs(outs[i].cpu().numpy() - ref).max()
        assert err <= 1e-5 * max(1.0, float(a.max() - a.min())), (i, a.shape, s, o, bc, err)
    plan.close()


def test_batch_stalled_copy_times_out_and_the_context_stays_usable(cuda):
    """A copy that never lands: with INJECT_STALLED_COPY the row-march launch announces its TMA copies
    without issuing them, so its bounded waits give up after a short limit; the launch reports
    DIPCU_ERR_TIMEOUT through the device status word with nothing in flight, and the same context
    then runs a normal plan correctly (no GPU fault, no hang)."""
    from diplib_b200 import _abi
    from diplib_b200.batch import INJECT_STALLED_COPY, device_status
    device_status(clear=True)
    rng = np.random.default_rng(12)
    imgs = [rng.random(s, dtype=np.float32) for s in [(100, 128), (77, 260), (200, 64)]]   # rows TMA can address
    params = [(2.0, [0, 1], "mirror"), (4.0, [1, 0], "periodic"), (1.0, [2, 2], "add zeros")]
    plan, ins, outs = run_plan(imgs, params, graph=False, autotune=False, flags=INJECT_STALLED_COPY)
    assert plan.info()["kernels_per_run"] == 2                    # weights and the row-march launch
    assert device_status(clear=True) == _abi.ERR_TIMEOUT
    plan.close()
    plan, ins, outs = run_plan(imgs, params, graph=True, autotune=False)
    check_all(imgs, params, outs)
    assert device_status(clear=True) == 0
    plan.close()
