"""The benchmark's multi-rank plumbing on CPU: two gloo ranks agree on the
slowest rank's time and on the whole-job rate; the reference arm does no
work on ranks other than 0."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, device="cpu")
        out[rank] = (ms, bench.job_rate(1e9, 3, world, ms))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_gloo():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == out[1]
    ms, rate = out[0]
    assert ms == 15.0
    assert rate == pytest.approx(1e9 * 3 * 2 / 0.015)


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(7.5, 1) == 7.5
    assert bench.job_rate(10, 2, 1, 1000.0) == 20.0


def test_reference_arm_is_rank0_only(capsys):
    import bench

    class A:
        n, nt, groups, steps, warmup, gpus = 201, 1501, 4, 1, 0, 2
    assert bench.run_reference(A(), rank=1) is None
    assert capsys.readouterr().out == ""


def test_c1_reference_arm_line():
    """`bench.py --workload c1 --impl reference` on the host cores: one JSON
    line with the arm's keys (the reference's afd2dc, or the oracle port when
    the reference build is absent)."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "bench.py", "--workload", "c1", "--impl", "reference",
                          "--steps", "1", "--warmup", "0"], cwd=root, capture_output=True,
                         text=True, timeout=600, check=True).stdout
    lines = [json.loads(x) for x in out.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["unit"] == "Gpt/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "Gpt/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
