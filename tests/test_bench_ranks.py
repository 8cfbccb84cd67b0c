"""bench.py's multi-rank logic on CPU: two gloo ranks (127.0.0.1), each with
its own step time; both see the slowest rank's time and the whole-job value
counts the work of both replicas (weak scaling).  The reference arm on a
small stencil: exactly K timed steps, a named row sample when K full SpMVs
would exceed its time budget, and no line from other ranks."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 * (rank + 1)                       # rank 1 is the slow one
        m = bench.max_over_ranks(ms, ws, torch.device("cpu"))
        out[rank] = (m, bench.job_gflops(ws, 2.0e9, 100, m))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0][0] == out[1][0] == 20.0
    # 2 replicas x 100 steps x 2 GFLOP in 20 ms
    assert out[0][1] == pytest.approx(2 * 2.0 * 100 / 0.020)


def test_single_rank_is_a_no_op():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, 1, None) == 3.5
    assert bench.job_gflops(1, 1e9, 10, 1000.0) == pytest.approx(10.0)


def _reference_line(capsys, monkeypatch, budget, steps, warmup, rank=0):
    import argparse
    import json
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setattr(bench, "REF_ARM_SECONDS", budget)
    bench.run_reference(argparse.Namespace(grid=8, warmup=warmup, steps=steps, gpus=1), 1, rank)
    out = capsys.readouterr().out.strip()
    return json.loads(out.splitlines()[-1]) if out else None


def test_reference_arm_times_exactly_k_full_steps(capsys, monkeypatch):
    d = _reference_line(capsys, monkeypatch, 120.0, 7, 2)
    assert d["impl"] == "reference" and d["steps"] == 7 and d["warmup"] == 2
    assert d["cpu_baseline"]["sample"].startswith("full matrix per step")
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"] == d["cpu_baseline"]["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_reference_arm_samples_rows_when_k_steps_exceed_the_budget(capsys, monkeypatch):
    d = _reference_line(capsys, monkeypatch, 1e-9, 5, 1)
    assert d["steps"] == 5 and d["cpu_baseline"]["sample"].startswith("first ")
    assert "5 timed steps after 1 untimed" in d["cpu_baseline"]["sample"]


def test_reference_arm_other_ranks_print_nothing(capsys, monkeypatch):
    assert _reference_line(capsys, monkeypatch, 120.0, 3, 1, rank=1) is None


def test_reference_arm_never_loads_the_library():
    """The reference arm builds its input with the oracle's generator: after a
    full run, neither the package nor libbspmv.so is in the process, and its
    config is the one the library's arm prints."""
    import json
    import subprocess
    code = (
        "import sys, json, argparse\n"
        f"sys.path.insert(0, {str(ROOT)!r})\n"
        "import bench\n"
        "bench.run_reference(argparse.Namespace(grid=8, warmup=1, steps=2, gpus=1), 1, 0)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'pkg': 'benchsp_b200' in sys.modules, 'so': 'libbspmv' in maps}))\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout
    line, probe = [json.loads(s) for s in out.strip().splitlines()[-2:]]
    assert probe == {"pkg": False, "so": False}
    sys.path.insert(0, str(ROOT))
    import bench
    assert line["config"] == bench.headline_config(8, 1)
    assert line["config"]["n"] == 8 ** 3 * 4 and line["config"]["nnz"] == 22 ** 3 * 16


def test_gather_probe_choice_matches_the_array_size():
    """The SpMM gather roofline uses the probe of the same gather width whose
    buffer is closest in size (by ratio) to the gathered array."""
    sys.path.insert(0, str(ROOT))
    import bench
    gpk = {"w64_l2": {"buffer_mb": 64}, "w64_dram": {"buffer_mb": 2048},
           "w256_l2": {"buffer_mb": 64}, "w256_dram": {"buffer_mb": 2048},
           "w256_m256": {"buffer_mb": 256}, "w256_m512": {"buffer_mb": 512}}
    n = 1 << 20
    assert bench.probe_for(gpk, 64, n * 32 * 2) == "l2"          # B of 64 MB at N = 32
    assert bench.probe_for(gpk, 256, n * 128 * 2) == "m256"      # 256 MB at N = 128
    assert bench.probe_for(gpk, 256, n * 256 * 2) == "m512"      # 512 MB at N = 256
    assert bench.probe_for(gpk, 256, 3 << 30) == "dram"
    assert bench.probe_for(gpk, 256, 1 << 20) == "l2"
    with pytest.raises(KeyError):
        bench.probe_for(gpk, 8, 1 << 20)


def test_profile_summaries_run_committed_files_only():
    """Every command quoted in profiles/*.md runs bench.py (or the oracle's
    own programs) with a --profile mode bench.py accepts, and names no
    scratch file."""
    import re
    sys.path.insert(0, str(ROOT))
    src = (ROOT / "bench.py").read_text()
    choices = re.search(r'"--profile", choices=\[([^\]]*)\]', src, re.S).group(1)
    modes = set(re.findall(r'"([a-z0-9_]+)"', choices))
    texts = {p.name: p.read_text() for p in (ROOT / "profiles").glob("*.md")}
    assert texts
    for name, t in texts.items():
        assert "_work/" not in t, name
        for m in re.findall(r"python bench\.py --profile ([a-z0-9_]+)", t):
            assert m in modes, (name, m)
        for script in re.findall(r"python ([A-Za-z0-9_/.]+\.py)", t):
            assert (ROOT / script).exists(), (name, script)
