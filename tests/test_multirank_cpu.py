"""The N>1 plumbing of bench.py on CPU: two ranks over gloo (127.0.0.1).  The
workloads are weak-scaled replicas (no data-path collective), so what has to
hold across ranks is the timing rule — the job's step time is the slowest
rank's — and the whole-job throughput built from it; the reference arm runs
on rank 0 only and the other ranks exit without work."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as td
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 * (rank + 1)  # rank 1 is the slow one
        rate, ms_max = bench.job_rate(torch, 1000, ms, td, world, device="cpu")
        td.barrier()
        out.put((rank, rate, ms_max))
    finally:
        td.destroy_process_group()


def test_job_rate_takes_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get() for _ in range(world))
    for rank, rate, ms_max in got:
        assert ms_max == 20.0  # the max over ranks, on every rank
        assert rate == pytest.approx(1000 * world / 0.020)


def test_job_rate_single_process():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    rate, ms = bench.job_rate(torch, 500, 4.0, None, 1, device="cpu")
    assert (rate, ms) == (500 / 0.004, 4.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = type("Args", (), {"workload": "tc14", "steps": 1, "warmup": 1, "gpus": 2})()
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.main_reference(args)
    assert buf.getvalue() == ""
    # rank 0 of the same job prints the line (k-truss: its documented unavailable line)
    monkeypatch.setenv("RANK", "0")
    args.workload = "ktruss20"
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.main_reference(args)
    line = json.loads(buf.getvalue())
    assert line["impl"] == "reference" and "unavailable" in line


def test_roofline_traffic_scales_with_streamed_entries():
    sys.path.insert(0, ROOT)
    import bench
    rec = json.load(open(os.path.join(ROOT, "profiles", "tc_rmat22_dram.json")))["6"]
    captured = rec["dram_read"] + rec["dram_write"]
    assert bench.traffic_for(6, rec["work"]) == captured  # the captured launch itself
    assert bench.traffic_for(6, rec["work"] * 16) == pytest.approx(captured * 16, rel=1e-9)
    assert bench.traffic_for(3, 10) is None  # no capture of that kernel (it ran no rows)


def test_clock_sampler_parses_nvidia_smi_lines(tmp_path, monkeypatch):
    """The clock sampler reads nvidia-smi's CSV from a pipe; a stand-in
    executable prints two samples, one of them with sw_power_cap active."""
    fake = tmp_path / "nvidia-smi"
    fake.write_text("#!/bin/sh\n"
                    "echo '0, 1965, 1965, 700.5, 0x0, Not Active, Not Active, Not Active, Not Active'\n"
                    "echo '0, 1800, 1965, 990.1, 0x4, Not Active, Not Active, Not Active, Active'\n"
                    "exec sleep 30\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}:{os.environ['PATH']}")
    sys.path.insert(0, ROOT)
    import time

    import bench
    c = bench.ClockSampler(0)
    c.start()
    time.sleep(0.5)
    got = c.stop()
    assert got == {"sm_mhz": 1882.5, "sm_max_mhz": 1965.0, "samples": 2, "reasons": ["sw_power_cap"]}


def test_reference_arm_on_a_small_workload(monkeypatch):
    """`bench.py --impl reference` on triangle counting RMAT-14: the sampled
    reference rows (never an empty sample, which the reference's mxmm_msa
    cannot take) give a positive rate and the contract's keys."""
    sys.path.insert(0, ROOT)
    import bench
    import oracle
    if not oracle.ref_available():
        pytest.skip("reference oracle not built")
    monkeypatch.setenv("RANK", "0")
    monkeypatch.setenv("WORLD_SIZE", "1")
    args = type("Args", (), {"workload": "tc14", "steps": 2, "warmup": 1, "gpus": 1})()
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.main_reference(args)
    line = json.loads(buf.getvalue())
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "edges/s"
    assert line["cpu_baseline"]["kind"] == "reference" and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["config"] == bench.tc_config(bench.WORKLOADS["tc14"], 16384, line["config"]["nnz_lower"])


def test_reference_arm_does_not_load_the_product_library():
    """The reference arm generates its input with the oracle's restatement of
    the generator: libgk_b200.so is never mapped into its process."""
    import subprocess
    code = ("import runpy, sys, os; os.environ['RANK'] = '0'; os.environ['WORLD_SIZE'] = '1'; "
            "sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'tc14', '--steps', '1', '--warmup', '0']; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "print('MAPPED', 'libgk_b200' in open('/proc/self/maps').read())")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "MAPPED False" in out.stdout and '"impl": "reference"' in out.stdout
