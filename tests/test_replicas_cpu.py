"""The multi-process path of bench.py on CPU (gloo, world size 2): bench.py runs one independent
replica per GPU ("replicas only": the filter has no cross-GPU exchange), and the only collective
steps are the barrier around the timed region and the max over ranks of its time.  Two gloo
ranks check that every rank receives the largest time, and that the reference arm on a rank
other than 0 exits 0 without work or output."""
from __future__ import annotations

import datetime
import io
import multiprocessing as mp
import os
import socket
import types
from contextlib import redirect_stdout


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m = bench._max_over_ranks(1.5 + rank, torch.device("cpu"))
        buf = io.StringIO()
        with redirect_stdout(buf):
            rc = bench.run_reference_arm(types.SimpleNamespace(steps=1, warmup=0, gpus=world)) if rank > 0 else 0
        dist.barrier()
        out.put((rank, m, rc, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time_and_only_rank0_reports():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[1] for r in res] == [2.5, 2.5]            # both ranks see the slowest rank's time
    assert res[1][2] == 0 and res[1][3] == ""            # rank 1: reference arm exits 0, prints nothing
    assert bench_single_process_max() == 3.0


def bench_single_process_max() -> float:
    """Without a process group the helper returns its argument."""
    import torch
    import bench
    return bench._max_over_ranks(3.0, torch.device("cpu"))


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` times the compiled reference on the host cores and prints one
    JSON line with the headline's metric, unit and workload, `impl`, a `cpu_baseline` describing
    the run and an `e2e` with no host-device traffic (or an `unavailable` line without the
    reference build)."""
    import json
    import subprocess
    import sys

    import oracle
    from tests.conftest import ROOT
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if not oracle.ref_available():
        assert "unavailable" in d
        return
    import bench
    assert d["metric"] == bench.METRIC and d["unit"] == "Gvox/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["config"]["workload"] == bench.CONFIG["workload"]
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
