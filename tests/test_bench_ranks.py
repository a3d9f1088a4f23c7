"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2).

bench.py runs one independent replica per GPU (the RBE + RBL step has no
exchange between replicas), synchronises the ranks with a barrier around the
timed region and reports the slowest rank's device time.  Here the same
helpers run as two gloo ranks on the host; the reference arm's rank handling
runs as two plain processes.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        # each rank's "device time" differs; every rank must see the largest
        ms = bench.max_over_ranks(10.0 + 3.0 * rank, ws, "cpu")
        value = bench.job_throughput(ws, 1000, 4, ms)
        with open(os.path.join(out, f"rank{rank}.json"), "w") as f:
            json.dump({"ms": ms, "value": value}, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    ws = 2
    mp.start_processes(_rank_main, args=(ws, _free_port(), str(tmp_path)), nprocs=ws,
                       join=True, start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(ws)]
    for r in res:
        assert r["ms"] == 13.0
        assert r["value"] == pytest.approx(2 * 1000 * 4 / 0.013)


def test_single_rank_helpers():
    assert bench.max_over_ranks(7.5, 1, "cpu") == 7.5
    assert bench.job_throughput(1, 200000, 50, 1000.0) == pytest.approx(1e7)
    assert bench.job_throughput(4, 200000, 50, 1000.0) == pytest.approx(4e7)


def _run_reference_arm(rank, ws):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank),
               MASTER_ADDR="127.0.0.1")
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                           "--gpus", str(ws), "--n", "1500", "--steps", "1", "--warmup", "3"],
                          capture_output=True, text=True, env=env, timeout=600)


def test_reference_arm_rank0_prints_line():
    r = _run_reference_arm(0, 2)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["unit"] == bench.UNIT
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"


def test_reference_arm_other_ranks_exit_quietly():
    r = _run_reference_arm(1, 2)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
