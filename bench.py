"""Benchmark of the SpMV hot path on B200.

Headline workload (one JSON line on rank 0): FP64 BSR SpMV, 4x4 blocks, on
the 3-D 27-point stencil over a 64^3 grid with 4 unknowns per node
(n = 1,048,576, 6,859,000 dense blocks, 109,744,000 nonzeros), x uniform in
[-1, 1].  One step = one y = A*x over the whole matrix with A, x, y resident
in HBM; the working set (923 MB) is larger than L2 (126 MB), so no flush is
needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun) runs N independent replicas, one per GPU (SpMV on one
matrix does not shard here); value = the work of all ranks / the slowest
rank's time.  --impl reference times the reference's own CPU SpMV
(ref_spmv_fp64, src/ref.cpp:26, compiled into oracle/_ref) on all host cores.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

GRID, DOF, SEED = 64, 4, 20261203 + 1
METRIC = "SpMV GFLOP/s (FP64 BSR 4x4, 27-pt stencil 64^3 x 4 dof)"
WORKLOAD = "bsr4_fp64_spmv_stencil27_64cubed_4dof"
E2E_CHUNKS = 8
# untimed warm-up of the host-buffer path: in a fresh process its first few
# hundred calls ran up to 1.5x slower (host copies not yet at full speed)
E2E_WARM_SECONDS = 0.25


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "src": "measured"}
    return {"hbm_gbs": 6650.0, "src": "fallback"}


def algorithmic_bytes_bsr(nb: int, blc_row: int, n: int, bs: int = 4) -> int:
    """Each array read or written once: values nb*bs^2*8, block columns nb*4,
    block-row pointers (blc_row+1)*4, x n*8, y n*8."""
    return nb * bs * bs * 8 + nb * 4 + (blc_row + 1) * 4 + n * 8 + n * 8


def max_over_ranks(ms: float, ws: int, device) -> float:
    """The slowest rank's time: every rank passes its own CUDA-event time;
    all ranks return the maximum (a no-op for one rank)."""
    if ws <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gflops(ws: int, flops_per_step: float, steps: int, ms: float) -> float:
    """Whole-job throughput of `ws` replicas that each ran `steps` steps of
    `flops_per_step`, over the slowest rank's time `ms` (weak scaling)."""
    return ws * flops_per_step * steps / (ms / 1e3) / 1e9


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.tmp, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.tmp.flush()
        lines = [ln.strip() for ln in Path(self.tmp.name).read_text().splitlines() if ln.strip()]
        os.unlink(self.tmp.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        # under load = samples in the upper half of the observed range
        load = [s for s in sm if sm and s >= 0.5 * max(sm)]
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_uuid(dev: int) -> str:
    import torch
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(dev)


# ---------------------------------------------------------------------------
# CPU reference: ref_spmv_fp64 (src/ref.cpp:26-37) on disjoint row ranges,
# one thread per core (ctypes releases the GIL during the call).

def _cpu_spmv(A, x):
    """The reference's CPU SpMV (`ref_spmv_fp64` compiled from src/ref.cpp,
    else the oracle's restatement) with the rows split evenly over every
    host core: returns (step, cores, kind, y), step(r_end) computing rows
    [0, r_end) of y = A x once."""
    sys.path.insert(0, str(ROOT))
    from oracle import pyoracle
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    rp64 = A.rowptr.astype(np.int64)
    ci64 = A.colidx.astype(np.int64)
    y = np.empty(A.rows)
    ref_so = pyoracle.REF_DIR / "libref_host.so"
    if ref_so.exists():
        L = C.CDLL(str(ref_so))
        fn = L.ref_spmv_fp64_c
        fn.argtypes = [C.c_void_p] * 5 + [C.c_int64, C.c_int64]
        kind = "reference"
    else:
        L = pyoracle.orc()
        fn = None
        kind = "port"

    def run(r0, r1):
        if r1 <= r0:
            return
        rp = rp64[r0:]
        if fn is not None:
            fn(C.c_void_p(rp.ctypes.data), C.c_void_p(ci64.ctypes.data), C.c_void_p(A.values.ctypes.data),
               C.c_void_p(x.ctypes.data), C.c_void_p(y[r0:].ctypes.data), r1 - r0, A.cols)
        else:
            L.orc_spmv_f64(r1 - r0, C.c_void_p(rp.ctypes.data), C.c_void_p(ci64.ctypes.data),
                           C.c_void_p(A.values.ctypes.data), C.c_void_p(x.ctypes.data),
                           C.c_void_p(y[r0:].ctypes.data))

    def step(r_end):
        bounds = np.linspace(0, r_end, cores + 1).astype(np.int64)
        ths = [threading.Thread(target=run, args=(int(bounds[t]), int(bounds[t + 1]))) for t in range(cores)]
        for th in ths:
            th.start()
        for th in ths:
            th.join()

    return step, cores, kind, y


def cpu_reference(A, x, max_seconds: float = 12.0, min_reps: int = 2) -> dict:
    """Median time of full CPU SpMVs (at least min_reps, at most 50, about
    max_seconds)."""
    step, cores, kind, y = _cpu_spmv(A, x)
    times = []
    t_start = time.perf_counter()
    while len(times) < min_reps or (time.perf_counter() - t_start < max_seconds and len(times) < 50):
        t0 = time.perf_counter()
        step(A.rows)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return {"gflops": 2.0 * A.nnz / t / 1e9, "cores": cores, "kind": kind, "reps": len(times),
            "seconds_per_spmv": t, "y": y}


def make_matrix(grid: int = GRID):
    import benchsp_b200 as bsp
    A = bsp.gen_stencil27(grid, DOF, SEED)
    x = bsp.gen_uniform(A.cols, SEED + 1)
    return A, x


def make_matrix_reference(grid: int = GRID):
    """The same matrix and x as make_matrix, built by the oracle's copy of the
    generator (bit-identical, checked in tests/test_generators.py), so the
    reference arm's process never loads the library."""
    from types import SimpleNamespace

    from oracle import pyoracle
    rp, ci, va = pyoracle.gen_stencil27(grid, DOF, SEED)
    n = rp.size - 1
    A = SimpleNamespace(rows=n, cols=n, nnz=int(ci.size), rowptr=rp, colidx=ci, values=va)
    return A, pyoracle.gen_uniform(n, SEED + 1)


def headline_config(grid: int, n_gpus: int) -> dict:
    """The workload's `config`, printed identically by both arms.  With 4
    unknowns per node every node is one 4x4 block row and couples to each of
    its neighbours by one dense block: (3*grid - 2)^3 blocks."""
    blocks = (3 * grid - 2) ** 3
    return {"workload": WORKLOAD if grid == GRID else f"bsr4_fp64_spmv_stencil27_{grid}cubed_4dof",
            "n": grid ** 3 * DOF, "nnz": blocks * DOF * DOF, "blocks": blocks, "block": "4x4",
            "parallelism": f"replicas{n_gpus}",
            "l2": f"inputs larger than L2 ({algorithmic_bytes_bsr(blocks, grid ** 3, grid ** 3 * DOF) / 1e6:.0f} MB "
                  f"working set)"}


def scaled_bsr_extra(M, x, steps: int, flops: float) -> dict:
    """The headline SpMV on the matrix stored as FP16 / BF16 values with one
    power-of-two scale per 4x4 block (FP32 products and sums, FP64 x and y):
    CUDA-event time per launch over `steps` launches after 3 untimed, and the
    stored bytes it moves (values 32 B + key 4 B per block, block-row
    pointers, x and y) per second against the HBM peak."""
    import torch
    out = {}
    pk = peaks()
    y = torch.empty(M.row, dtype=torch.float64, device=x.device)
    for dt in ("f16", "bf16"):
        S = M.scaled(dt)
        for _ in range(3):
            S.spmv(x, y)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            S.spmv(x, y)
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / steps / 1e3
        nbytes = S.stored_bytes() + 8 * (M.row + M.col)
        out[dt] = {"us": round(t * 1e6, 2), "gflops": round(flops / t / 1e9, 1), "bytes_per_launch": nbytes,
                   "gbs": round(nbytes / t / 1e9, 1), "frac": round(nbytes / t / 1e9 / pk["hbm_gbs"], 4)}
        S.free()
    return out


def cg_poisson128(bsp, dev, grid: int = 128, reps: int = 3) -> dict:
    """CG to 1e-10 on the 7-point Poisson matrix 128^3 (b uniform [-1, 1]) in
    FP64 and with FP32, FP16 and BF16 stored values (FP64 residual, dots and
    update): per mode the median wall time of `reps` solves after one untimed
    solve (CUDA events inside the solver), iterations, and ||b - A x|| / ||b||
    recomputed in FP64 by cuSPARSE (torch.sparse), independent of the solver."""
    import torch
    A = bsp.gen_poisson3d(grid)
    bh = bsp.gen_uniform(A.rows, SEED + 3)
    rp, ci, va, b = (torch.from_numpy(a).to(dev) for a in (A.rowptr, A.colidx, A.values, bh))
    T = torch.sparse_csr_tensor(rp.long(), ci.long(), va, size=(A.rows, A.cols))
    out = {"n": A.rows, "nnz": A.nnz, "tol": 1e-10}
    for mode in ("fp64", "f32", "f16", "bf16"):
        S = bsp.CgSolver(rp, ci, va, mode=mode, tol=1e-10)
        S.solve(b)
        runs = []
        for _ in range(reps):
            xs, r = S.solve(b)
            runs.append((r["seconds"], r, xs))
        runs.sort(key=lambda t: t[0])
        sec, r, xs = runs[len(runs) // 2]
        res = float(torch.linalg.norm(b - T @ xs) / torch.linalg.norm(b))
        out[mode] = {"ms": round(sec * 1e3, 3), "iterations": r["iterations"], "rel_residual_fp64": res,
                     "converged": bool(r["converged"]) and res <= 1e-10}
        S.close()
    best = min(("f32", "f16", "bf16"), key=lambda m: out[m]["ms"])
    out["fastest_mixed"] = best
    out["mixed_over_fp64_time"] = round(out[best]["ms"] / out["fp64"]["ms"], 4)
    return out


REF_ARM_SECONDS = 120.0   # the reference arm's K timed steps together


def run_reference(args, ws, rank):
    """The reference's CPU path on this workload: W untimed steps, then
    exactly K timed steps.  A step is one SpMV over the full matrix, or over
    its first rows when K full SpMVs would take longer than REF_ARM_SECONDS
    (the sample is named in the line); GFLOP/s = 2 * sample nnz * K / time."""
    if rank != 0:
        return
    A, x = make_matrix_reference(args.grid)
    step, cores, kind, _ = _cpu_spmv(A, x)
    warm = []
    for _ in range(max(1, args.warmup)):
        t0 = time.perf_counter()
        step(A.rows)
        warm.append(time.perf_counter() - t0)
    t_full = statistics.median(warm)
    k = max(1, args.steps)
    rows = A.rows
    if k * t_full > REF_ARM_SECONDS:
        rows = max(cores, int(A.rows * REF_ARM_SECONDS / (k * t_full)))
    nnz = int(A.rowptr[rows]) - int(A.rowptr[0])
    t0 = time.perf_counter()
    for _ in range(k):
        step(rows)
    total = time.perf_counter() - t0
    v = 2.0 * nnz * k / total / 1e9
    sample = (f"full matrix per step ({A.rows} rows, {A.nnz} nonzeros)" if rows == A.rows else
              f"first {rows} of {A.rows} rows per step ({nnz} nonzeros)")
    sample += f", {k} timed steps after {max(1, args.warmup)} untimed, rows split over {cores} threads"
    line = {
        "metric": METRIC, "value": round(v, 3), "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": k,
        "warmup": args.warmup, "ms_per_step": round(total / k * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": headline_config(args.grid, args.gpus),
        "impl": "reference",
        "cpu_baseline": {"value": round(v, 3), "unit": "GFLOP/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": round(v, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, ws, rank, local):
    import torch

    import benchsp_b200 as bsp
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    A, x_h = make_matrix(args.grid)
    rp, ci, va = (torch.from_numpy(a).to(dev) for a in (A.rowptr, A.colidx, A.values))
    x = torch.from_numpy(x_h).to(dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=4)
    torch.cuda.synchronize()
    convert_s = time.perf_counter() - t0
    del rp, ci, va
    torch.cuda.empty_cache()
    y = torch.empty(A.rows, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()
    flops = 2.0 * A.nnz
    algo_bytes = algorithmic_bytes_bsr(M.blc_num, M.blc_row, A.rows)

    for _ in range(max(args.warmup, 3)):
        M.spmv(x, y)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_uuid(local)) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            M.spmv(x, y)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), ws, dev)
    if ws > 1:
        torch.distributed.barrier()
    ms_step = ms / args.steps
    value = job_gflops(ws, flops, args.steps, ms)

    # e2e through the host-buffer C-ABI call: H2D x, SpMV, D2H y per step
    xh = torch.from_numpy(x_h).pin_memory()
    yh = torch.empty(A.rows, dtype=torch.float64).pin_memory()
    xh_np, yh_np = xh.numpy(), yh.numpy()
    e2e_steps = max(3, min(args.steps, 200))
    HP = M.host_plan(E2E_CHUNKS)   # overlapped x upload / SpMV / y download
    t_warm = time.perf_counter()
    n_warm = 0
    while n_warm < max(3, args.warmup) or time.perf_counter() - t_warm < E2E_WARM_SECONDS:
        HP.spmv(xh_np, yh_np)
        n_warm += 1
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        HP.spmv(xh_np, yh_np)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), ws, dev)
    e2e_value = job_gflops(ws, flops, e2e_steps, e2e_ms)

    # correctness of the benchmarked result (cheap, outside the timed region)
    y_np = y.cpu().numpy()
    ok = bool(np.allclose(y_np, yh_np, rtol=0, atol=0))

    # the same matrix with FP16/BF16 values and one power-of-two scale per block
    scaled = scaled_bsr_extra(M, x, args.steps, flops)

    # the CG target (mixed precision vs FP64 to 1e-10), outside the timed region
    cg = cg_poisson128(bsp, dev) if (ws == 1 and not args.no_cg) else None

    if rank != 0:
        return
    cfg = headline_config(args.grid, ws)
    assert (cfg["n"], cfg["nnz"], cfg["blocks"]) == (A.rows, A.nnz, M.blc_num), "config does not describe the matrix"
    pk = peaks()
    achieved = algo_bytes / (ms_step / 1e3) / 1e9
    traffic = None
    tp = ROOT / "profiles" / "bsr4_ffma_stencil27_traffic.json"
    if tp.exists():
        traffic = json.loads(tp.read_text()).get("dram_bytes_per_launch")
    cpu = None
    if ws == 1 and not args.no_cpu_baseline:
        ref = cpu_reference(A, x_h, max_seconds=10.0)
        rel = float(np.max(np.abs(ref["y"] - y_np) / (np.abs(ref["y"]) + 1e-300)))
        cpu = {"value": round(ref["gflops"], 3), "unit": "GFLOP/s", "cores": ref["cores"], "kind": ref["kind"],
               "sample": f"full matrix (n={A.rows}, nnz={A.nnz}), median of {ref['reps']} SpMVs, rows split "
                         f"over {ref['cores']} threads", "max_rel_err_gpu_vs_cpu": rel}
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 6), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": cfg,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / pk["hbm_gbs"], 4), "traffic": traffic,
                     "peak_src": pk["src"], "algorithmic_bytes_per_launch": algo_bytes},
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_value, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 8 * A.cols,
                "d2h_bytes_per_step": 8 * A.rows, "steps": e2e_steps,
                "call": f"bsp_bsr_spmv_host_pipelined ({E2E_CHUNKS} chunks, pinned host x/y)"},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "extra": {"kernel": "bsr_ffma_kernel<4,16,1>", "csr2bsr_seconds": round(convert_s, 4),
                  "gbs": round(achieved, 1), "e2e_matches_device_result": ok, "scaled_16bit_bsr": scaled,
                  "cg_poisson128": cg},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# --suite: one JSON line per further workload (CSR Laplacian, BSR 8x8 and
# random-fill BSR, DASP on power-law rows, CG, SpMM on a power-law graph,
# batched SpMV).  Not part of the headline line; single GPU.

def _timed(fn, steps: int, flush=None) -> float:
    """Seconds per call, CUDA events on the current stream.  With `flush`, L2
    is overwritten between calls and only the calls themselves are timed."""
    import torch
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    if flush is None:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps / 1e3
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in evs:
        flush()
        a.record()
        fn()
        b.record()
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs) / steps / 1e3


def _timed_graph_flushed(fn, flush, reps: int = 50) -> float:
    """Seconds per call with L2 flushed before every call and no launch
    gaps: `reps` x (flush, call) captured in one CUDA graph, minus the same
    graph of flushes alone (CUDA events around each replay, best of 5)."""
    import torch
    fn()
    flush()
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    graphs = []
    for with_call in (True, False):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            for _ in range(reps):
                flush()
                if with_call:
                    fn()
        graphs.append(g)
    out = []
    for g in graphs:
        best = None
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            g.replay()
            e1.record()
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            best = t if best is None or t < best else best
        out.append(best)
    del graphs
    return (out[0] - out[1]) / reps


def _csr_bytes(rows: int, cols: int, nnz: int, vbytes: int = 8) -> int:
    return nnz * (vbytes + 4) + (rows + 1) * 4 + cols * vbytes + rows * vbytes


def _emit(name: str, **kw) -> None:
    print(json.dumps({"suite": name, **kw}), flush=True)


def _roof(nbytes: int, t: float, pk: float) -> dict:
    a = nbytes / t / 1e9
    return {"bound": "hbm", "achieved": round(a, 1), "peak": pk, "unit": "GB/s", "frac": round(a / pk, 4),
            "algorithmic_bytes": int(nbytes)}


def _cusparse_spmv(rp, ci, va, x, rows, cols):
    """torch.sparse CSR matvec (cuSPARSE) for comparison only."""
    import torch
    T = torch.sparse_csr_tensor(rp.long(), ci.long(), va, size=(rows, cols))
    return lambda: T @ x


def run_suite(args) -> None:
    import torch

    import benchsp_b200 as bsp
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    pk = peaks()["hbm_gbs"]
    scratch = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    flush = scratch.zero_
    steps = max(10, min(args.steps, 200))
    # bring the clocks up before the first (short) timed calls
    t_end = time.time() + 0.5
    while time.time() < t_end:
        for _ in range(50):
            flush()
        torch.cuda.synchronize()

    def up(*arrs):
        return [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in arrs]

    # --- CSR FP64 SpMV, 2-D Laplacian 512x512 (L2 flushed between calls)
    A = bsp.gen_laplace2d(512, 512)
    xh = bsp.gen_uniform(A.cols, SEED + 10)
    rp, ci, va, x = up(A.rowptr, A.colidx, A.values, xh)
    y = torch.empty(A.rows, dtype=torch.float64, device=dev)
    nb = _csr_bytes(A.rows, A.cols, A.nnz)
    ref = cpu_reference(A, xh, max_seconds=3.0)
    res = {}
    for algo in ("auto", "vector", "merge", "scalar"):
        t = _timed(lambda: bsp.csr_spmv(rp, ci, va, x, y, algo=algo), steps, flush)
        yy = y.cpu().numpy()
        res[algo] = {"us": round(t * 1e6, 2), "gflops": round(2 * A.nnz / t / 1e9, 2),
                     "bit_exact_vs_reference": bool(np.array_equal(yy, ref["y"])),
                     "max_rel_err": float(np.max(np.abs(yy - ref["y"]) / (np.abs(ref["y"]) + 1e-300)))}
    tcs = _timed(_cusparse_spmv(rp, ci, va, x, A.rows, A.cols), steps, flush)
    # the same calls replayed from a CUDA graph (no launch gaps), L2 flushed before each
    tg = _timed_graph_flushed(lambda: bsp.csr_spmv(rp, ci, va, x, y, algo="vector"), flush)
    res["vector_graph_replay"] = {"us": round(tg * 1e6, 2), "gflops": round(2 * A.nnz / tg / 1e9, 2),
                                  "roofline": _roof(nb, tg, pk)}
    _emit("csr_fp64_laplace2d_512", n=A.rows, nnz=A.nnz, l2="flushed between calls", variants=res,
          roofline=_roof(nb, res["auto"]["us"] / 1e6, pk), cusparse_us=round(tcs * 1e6, 2),
          cpu_baseline={"value": round(ref["gflops"], 3), "unit": "GFLOP/s", "cores": ref["cores"],
                        "kind": ref["kind"]})
    del rp, ci, va, x, y

    # --- BSR FP64: stencil 64^3 x 4 dof as 4x4 and 8x8 blocks; random-fill 4x4
    A, xh = make_matrix(GRID)
    rp, ci, va, x = up(A.rowptr, A.colidx, A.values, xh)
    y = torch.empty(A.rows, dtype=torch.float64, device=dev)
    tcs = _timed(_cusparse_spmv(rp, ci, va, x, A.rows, A.cols), steps)
    for bs in (4, 8):
        M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=bs)
        nb = algorithmic_bytes_bsr(M.blc_num, M.blc_row, A.rows, bs)
        res = {}
        for algo in (("auto", "ffma", "dmma") if bs == 4 else ("auto", "ffma")):   # DMMA: 4x4 blocks only
            t = _timed(lambda: M.spmv(x, y, algo=algo), steps)
            res[algo] = {"us": round(t * 1e6, 2), "gflops": round(2 * A.nnz / t / 1e9, 1),
                         "gbs": round(nb / t / 1e9, 1)}
        _emit(f"bsr{bs}_fp64_stencil27_64cubed_4dof", n=A.rows, nnz=A.nnz, blocks=M.blc_num,
              fill=round(A.nnz / (M.blc_num * bs * bs), 4), variants=res,
              roofline=_roof(nb, res["auto"]["us"] / 1e6, pk), cusparse_csr_us=round(tcs * 1e6, 2))
        M.free()
    del rp, ci, va, x, y
    torch.cuda.empty_cache()
    A = bsp.gen_random_bsr(262144, 4, 16, 0.3, 1.0, SEED + 11)
    xh = bsp.gen_uniform(A.cols, SEED + 12)
    rp, ci, va, x = up(A.rowptr, A.colidx, A.values, xh)
    y = torch.empty(A.rows, dtype=torch.float64, device=dev)
    M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=4)
    nb = algorithmic_bytes_bsr(M.blc_num, M.blc_row, A.rows, 4)
    res = {}
    for algo in ("auto", "ffma", "dmma", "adaptive"):
        t = _timed(lambda: M.spmv(x, y, algo=algo), steps)
        res[algo] = {"us": round(t * 1e6, 2), "gflops": round(2 * A.nnz / t / 1e9, 1), "gbs": round(nb / t / 1e9, 1)}
    tcs = _timed(_cusparse_spmv(rp, ci, va, x, A.rows, A.cols), steps)
    _emit("bsr4_fp64_random_16perrow_fill30to100", n=A.rows, nnz=A.nnz, blocks=M.blc_num,
          fill=round(A.nnz / (M.blc_num * 16), 4), variants=res, roofline=_roof(nb, res["auto"]["us"] / 1e6, pk),
          cusparse_csr_us=round(tcs * 1e6, 2))
    M.free()
    del rp, ci, va, x, y

    # --- DASP vs CSR on power-law rows (Zipf 2.0, capped at 10k, n = 2M)
    A = bsp.gen_powerlaw(1 << 21, 2.0, 10000, SEED + 13)
    xh = bsp.gen_uniform(A.cols, SEED + 14)
    rp, ci, va, x = up(A.rowptr, A.colidx, A.values, xh)
    y = torch.empty(A.rows, dtype=torch.float64, device=dev)
    D = bsp.csr2dasp(rp, ci, va, rows=A.rows, cols=A.cols)
    nb = _csr_bytes(A.rows, A.cols, A.nnz)
    res = {}
    for name, fn in (("dasp", lambda: D.spmv(x, y)), ("csr_auto", lambda: bsp.csr_spmv(rp, ci, va, x, y)),
                     ("csr_merge", lambda: bsp.csr_spmv(rp, ci, va, x, y, algo="merge"))):
        t = _timed(fn, steps)
        res[name] = {"us": round(t * 1e6, 2), "gflops": round(2 * A.nnz / t / 1e9, 1), "gbs": round(nb / t / 1e9, 1)}
    tcs = _timed(_cusparse_spmv(rp, ci, va, x, A.rows, A.cols), steps)
    _emit("dasp_fp64_powerlaw_2M_zipf2", n=A.rows, nnz=A.nnz, variants=res,
          roofline=_roof(nb, res["dasp"]["us"] / 1e6, pk), cusparse_us=round(tcs * 1e6, 2))
    D.free()
    del rp, ci, va, x, y

    # --- CG on the 7-point Poisson 128^3 to 1e-10: FP64 vs mixed precision
    A = bsp.gen_poisson3d(128)
    bh = bsp.gen_uniform(A.rows, SEED + 3)
    rp, ci, va, b = up(A.rowptr, A.colidx, A.values, bh)
    res = {}
    for mode in ("fp64", "f32", "f16", "bf16"):
        S = bsp.CgSolver(rp, ci, va, mode=mode, tol=1e-10)
        S.solve(b)
        best = None
        for _ in range(3):
            xs, r = S.solve(b)
            best = r if best is None or r["seconds"] < best["seconds"] else best
        res[mode] = {"ms": round(best["seconds"] * 1e3, 3), "iterations": best["iterations"],
                     "reliable_updates": best["reliable_updates"], "rel_residual": best["rel_residual"],
                     "gbs": round(best["bytes_moved"] / best["seconds"] / 1e9, 1)}
        S.close()
    _emit("cg_poisson3d_128_tol1e-10", n=A.rows, nnz=A.nnz, modes=res,
          mixed_speedup_vs_fp64=round(res["fp64"]["ms"] / min(res[m]["ms"] for m in ("f32", "f16", "bf16")), 3))
    del rp, ci, va, b

    # --- preconditioned CG: Jacobi / block-Jacobi on SPD matrices that need them
    run_pcg(bsp, up)

    # --- CG with 8 right-hand sides at once vs 8 single solves
    run_cg_multi(bsp, up, dev)

    # --- random-gather rate of this GPU (the ceiling of the gather-bound kernels)
    gpk = run_gather_peaks(bsp, dev)

    # --- SpMM on a power-law graph (n = 2^20, Zipf 1.8, mean degree 32)
    A = bsp.gen_graph(1 << 20, 1.8, 32, SEED + 4)
    rp, ci, v64 = up(A.rowptr, A.colidx, A.values)
    A64 = torch.sparse_csr_tensor(rp.long(), ci.long(), v64, size=(A.rows, A.cols))
    res = {}
    for name, tdt in (("f16", torch.float16), ("bf16", torch.bfloat16)):
        v = v64.to(tdt)
        P = bsp.SpmmPlan(rp, ci, v, cols=A.cols, chunk=256)
        for N in (32, 128, 256):
            g = torch.Generator(device="cpu").manual_seed(N)
            B = (torch.rand(A.cols, N, generator=g, dtype=torch.float64) * 2 - 1).to(tdt).to(dev)
            Cm = P.spmm(B)
            Cref = A64 @ B.double()
            err = float(torch.linalg.norm(Cm.double() - Cref) / torch.linalg.norm(Cref))
            t = _timed(lambda: P.spmm(B, Cm), 10)
            tg = _timed(lambda: P.spmm(B, Cm, engine="grouped"), 10)
            Af = torch.sparse_csr_tensor(rp.long(), ci.long(), v.float(), size=(A.rows, A.cols))
            Bf = B.float()
            tcs = _timed(lambda: Af @ Bf, 5)
            nb = A.nnz * 6 + (A.rows + 1) * 4 + A.cols * N * 2 + A.rows * N * 4
            gb = A.nnz * N * 2    # B-row bytes gathered (one B row per nonzero)
            w = min(256, 2 * N)
            where = probe_for(gpk, w, A.cols * N * 2)
            res[f"{name}_N{N}"] = {"ms": round(t * 1e3, 3), "engine": "slab", "grouped_engine_ms": round(tg * 1e3, 3),
                                   "gflops": round(2 * A.nnz * N / t / 1e9, 1),
                                   "rel_err_vs_fp64": err, "cusparse_f32_ms": round(tcs * 1e3, 3),
                                   "min_bytes_gbs": round(nb / t / 1e9, 1),
                                   "gather_roofline": {"bound": "random gathers", "achieved": round(gb / t / 1e9, 1),
                                                       "peak": gpk[f"w{w}_{where}"]["gbs"], "unit": "GB/s",
                                                       "frac": round(gb / t / 1e9 / gpk[f"w{w}_{where}"]["gbs"], 3),
                                                       "peak_src": f"bsp_gather_probe width {w} B, "
                                                                   f"{gpk[f'w{w}_{where}']['buffer_mb']} MB buffer"}}
        P.free()
    _emit("spmm_graph_1M_zipf1.8_deg32", n=A.rows, nnz=A.nnz, max_row=int(np.diff(A.rowptr).max()), variants=res)
    run_smat_graph(bsp, dev, up, A)
    del rp, ci, v64, A64
    run_gtile(bsp, dev, up, A, gpk)

    # --- block SpMM on dense 16x16 tiles: tcgen05 vs mma.sync vs CSR
    A = bsp.gen_random_bsr(32768, 16, 8, 1.0, 1.0, SEED + 5)
    rp, ci, v64 = up(A.rowptr, A.colidx, A.values)
    res = {}
    for name, tdt in (("f16", torch.float16), ("bf16", torch.bfloat16)):
        M = bsp.SmatMatrix(rp, ci, v64, rows=A.rows, cols=A.cols, dtype=name)
        v = v64.to(tdt)
        for N in (32, 64, 128, 256):
            B = (torch.rand(A.cols, N, generator=torch.Generator().manual_seed(N)) * 2 - 1).to(tdt).to(dev)
            Cref = torch.sparse_csr_tensor(rp.long(), ci.long(), v64, size=(A.rows, A.cols)) @ B.double()
            row = {}
            for path in ("tcgen05", "tcgen05_w64", "tcgen05_w128", "tcgen05_persistent", "tcgen05_persistent_w64", "mma_sync"):
                Cm = M.spmm(B, path=path)
                err = float(torch.linalg.norm(Cm.double() - Cref) / torch.linalg.norm(Cref))
                t = _timed(lambda: M.spmm(B, Cm, path=path), 10)
                row[path] = {"ms": round(t * 1e3, 4), "tflops": round(2 * A.nnz * N / t / 1e12, 2),
                             "rel_err_vs_fp64": err}
            t = _timed(lambda: bsp.spmm_csr(rp, ci, v, B), 5)
            row["csr_grouped"] = {"ms": round(t * 1e3, 4), "tflops": round(2 * A.nnz * N / t / 1e12, 2)}
            res[f"{name}_N{N}"] = row
        M.check()
        M.free()
    _emit("smat_dense16_tiles_524k_rows_8_per_row", rows=A.rows, nnz=A.nnz, tiles=A.nnz // 256, variants=res)
    del rp, ci, v64

    # --- per-block scaled FP16/BF16 BSR on the headline matrix
    run_scaled_bsr(bsp, dev, pk, up)

    # --- 512 independent SpMVs (and 8-RHS SpMMs) in one persistent launch
    run_batch(bsp, dev, pk, up)

    # --- Matrix Market file -> CSR (stencil 32^3 x 4 dof written by the library)
    run_mtx_read(bsp, dev)

    # --- row-similarity reordering of a row-shuffled tile matrix
    run_reorder_similarity(bsp, dev, up)


def run_gather_peaks(bsp, dev) -> dict:
    """bsp_gather_probe: random gathers of 8 B (a CSR/DASP x gather), 64 B
    and 256 B (B-row slices of the SpMM) from a buffer that fits L2 (16 or 64
    MB) and from one that does not (2 GB), and 256 B from 256 and 512 MB (the
    sizes of the SpMM's B at N = 128 and 256, partly in L2); 10 timed
    launches after 3."""
    import torch
    out = {}
    for width, count in ((8, 50_000_000), (64, 33_554_432), (256, 33_554_432)):
        sizes = [("l2", 16 if width == 8 else 64), ("dram", 2048)]
        if width == 256:
            sizes += [("m256", 256), ("m512", 512)]
        for where, mb in sizes:
            buf = torch.zeros((mb << 20) // 4, dtype=torch.int32, device=dev)
            t = _timed(lambda: bsp.gather_probe(buf, width, count), 10)
            out[f"w{width}_{where}"] = {"buffer_mb": mb, "ggathers_s": round(count / t / 1e9, 2),
                                        "gbs": round(count * width / t / 1e9, 1)}
            del buf
    _emit("gather_probe", variants=out)
    return out


def probe_for(gpk: dict, width: int, nbytes: float) -> str:
    """The gather-probe entry of this width whose buffer is closest in size
    (by ratio) to a gathered array of `nbytes` bytes: its key suffix."""
    cands = [k for k in gpk if k.startswith(f"w{width}_")]
    if not cands:
        raise KeyError(f"no gather probe of width {width}")
    mb = max(nbytes / 2 ** 20, 1e-9)
    best = min(cands, key=lambda k: abs(np.log(gpk[k]["buffer_mb"] / mb)))
    return best.split("_", 1)[1]


def run_smat_graph(bsp, dev, up, A) -> None:
    """The SMaT tensor-core path on the power-law graph itself: rows
    regrouped by row similarity (host, one-time), 16x16 tiles of the
    reordered rows, tcgen05 SpMM at N = 32 / 128 / 256 (FP16), beside the
    slab CSR engine on the same rows; the engine choice's estimates."""
    import time

    import torch
    t0 = time.perf_counter()
    perm = bsp.reorder_similarity_host(A.rowptr, A.colidx, A.cols)
    reorder_s = time.perf_counter() - t0
    R = bsp.permute_rows_csr_host(A, perm)
    choice, _ = bsp.choose_spmm_host(R, 128, reorder=False)
    rp, ci, va = up(R.rowptr, R.colidx, R.values)
    try:
        Sm = bsp.SmatMatrix(rp, ci, va, rows=R.rows, cols=R.cols, dtype="f16")
    except bsp.BspError as ex:
        # 16x16 tiles of this graph hold more than 2^31 stored entries
        _emit("smat_tcgen05_graph_1M_reordered", rows=R.rows, nnz=R.nnz, reorder_host_s=round(reorder_s, 2),
              tiles=choice["tiles_given"], tile_fill=round(R.nnz / (256.0 * choice["tiles_given"]), 4),
              tile_bytes_f16=choice["tiles_given"] * 512, csr_bytes_f16=R.nnz * 6 + 4 * (R.rows + 1),
              unavailable=str(ex), chooser=choice["engine"])
        return
    P = bsp.SpmmPlan(rp, ci, va.half(), cols=R.cols, chunk=256)
    res = {}
    for N in (32, 128, 256):
        B = (torch.rand(R.cols, N, generator=torch.Generator().manual_seed(N)) * 2 - 1).half().to(dev)
        Ct = Sm.spmm(B, path="tcgen05")
        Cs = P.spmm(B)
        t = _timed(lambda: Sm.spmm(B, Ct, path="tcgen05"), 5)
        ts = _timed(lambda: P.spmm(B, Cs), 5)
        rel = float(torch.linalg.norm(Ct.double() - Cs.double()) / torch.linalg.norm(Cs.double()))
        cN, _ = bsp.choose_spmm_host(R, N, reorder=False)
        res[f"N{N}"] = {"smat_tcgen05_ms": round(t * 1e3, 3), "slab_csr_ms": round(ts * 1e3, 3),
                        "tflops_tcgen05": round(2 * R.nnz * N / t / 1e12, 3), "rel_diff_tc_vs_csr": rel,
                        "chooser": cN["engine"]}
    Sm.check()
    _emit("smat_tcgen05_graph_1M_reordered", rows=R.rows, nnz=R.nnz, reorder_host_s=round(reorder_s, 2),
          tiles=Sm.tiles, tile_fill=round(Sm.fill, 4), variants=res)
    Sm.free()
    P.free()


def _permute_columns(A, seed: int):
    """A with its columns renumbered by a seeded random permutation (each
    row's entries re-sorted by the new column)."""
    perm = np.random.default_rng(seed).permutation(A.cols).astype(np.int32)
    rows = np.repeat(np.arange(A.rows, dtype=np.int32), np.diff(A.rowptr))
    nc = perm[A.colidx]
    o = np.lexsort((nc, rows))
    return type(A)(A.rows, A.cols, A.rowptr, np.ascontiguousarray(nc[o]), np.ascontiguousarray(A.values[o]))


def run_gtile(bsp, dev, up, graph, gpk) -> None:
    """Gathered-tile tcgen05 SpMM (bsp_gtile: every 16-row group's distinct
    columns in chunks of 16 with their 16x16 value tiles, the chunk's B rows
    gathered into shared memory) beside the slab CSR engine, FP16, N = 32 /
    128 / 256: a 27-point stencil 48^3 x 4 dof with its columns permuted at
    random (a group's rows share columns scattered over the whole range, so
    the matrix's own 16x16 tiles are nearly empty while its chunks are half
    full) and the power-law graph (chunks about 1/16 full).  The engine
    choice's pick and estimates; the product against torch.sparse FP64 on
    the same FP16 values."""
    import time

    import torch
    for label, A in (("stencil27_48cubed_4dof_columns_permuted", _permute_columns(make_matrix(48)[0], SEED + 7)),
                     ("graph_1M_zipf1.8_deg32", graph)):
        rp, ci, v64 = up(A.rowptr, A.colidx, A.values)
        vh = v64.half()
        Ah = bsp.HostCSR(A.rows, A.cols, A.rowptr, A.colidx, vh.double().cpu().numpy())
        t0 = time.perf_counter()
        G = bsp.GatherTileMatrix(Ah, "f16")
        build_s = time.perf_counter() - t0
        chunks = int(G.nchunks)
        A64 = torch.sparse_csr_tensor(rp.long(), ci.long(), vh.double(), size=(A.rows, A.cols))
        P = bsp.SpmmPlan(rp, ci, vh, cols=A.cols, chunk=256)
        res = {}
        for N in (32, 128, 256):
            g = torch.Generator(device="cpu").manual_seed(N)
            B = (torch.rand(A.cols, N, generator=g, dtype=torch.float64) * 2 - 1).half().to(dev)
            Cg = G.spmm(B)
            Cs = P.spmm(B)
            Cref = A64 @ B.double()
            err = float(torch.linalg.norm(Cg.double() - Cref) / torch.linalg.norm(Cref))
            tg = _timed(lambda: G.spmm(B, Cg), 10)
            ts = _timed(lambda: P.spmm(B, Cs), 10)
            choice, _ = bsp.choose_spmm_host(A, N, reorder=False)
            gathered = chunks * 16 * N * 2
            w = min(256, 2 * N)
            res[f"N{N}"] = {"gtile_ms": round(tg * 1e3, 3), "slab_csr_ms": round(ts * 1e3, 3),
                            "speedup_vs_slab": round(ts / tg, 2), "tflops": round(2 * A.nnz * N / tg / 1e12, 2),
                            "rel_err_vs_fp64": err, "chooser": choice["engine"],
                            "est_ms": {"gtile": round(choice["est_seconds_gtile_given"] * 1e3, 3),
                                       "csr": round(choice["est_seconds_csr"] * 1e3, 3)},
                            "gather_roofline": {"bound": "random gathers", "achieved": round(gathered / tg / 1e9, 1),
                                                "peak": gpk[f"w{w}_dram"]["gbs"], "unit": "GB/s",
                                                "frac": round(gathered / tg / 1e9 / gpk[f"w{w}_dram"]["gbs"], 3),
                                                "peak_src": f"bsp_gather_probe width {w} B, "
                                                            f"{gpk[f'w{w}_dram']['buffer_mb']} MB buffer"}}
        G.check()
        _emit(f"gtile_spmm_{label}", rows=A.rows, nnz=A.nnz, build_host_s=round(build_s, 2), chunks=chunks,
              chunk_fill=round(A.nnz / (256.0 * chunks), 4), tiles_16x16=choice["tiles_given"],
              tile_fill=round(A.nnz / (256.0 * choice["tiles_given"]), 4), variants=res)
        G.free()
        P.free()
        del rp, ci, v64, vh, A64


def run_scaled_bsr(bsp, dev, pk, up) -> None:
    """FP64 BSR against the FP16/BF16 per-block-scaled copy on the stencil
    64^3 x 4 dof, 4x4 and 8x8 blocks, FP64 and FP32 x/y; roofline on the
    stored bytes."""
    import torch
    A, xh = make_matrix(GRID)
    rp, ci, va, x = up(A.rowptr, A.colidx, A.values, xh)
    y = torch.empty(A.rows, dtype=torch.float64, device=dev)
    x32, y32 = x.float(), torch.empty(A.rows, dtype=torch.float32, device=dev)
    res = {}
    for bs in (4, 8):
        M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=bs)
        t64 = _timed(lambda: M.spmv(x, y), 20)
        row = {"fp64_us": round(t64 * 1e6, 2)}
        for dt in ("f16", "bf16"):
            S = M.scaled(dt)
            for xy, xx, yy, vb in (("f64xy", x, y, 8), ("f32xy", x32, y32, 4)):
                t = _timed(lambda: S.spmv(xx, yy), 20)
                nb = S.stored_bytes() + vb * (A.rows + A.cols)
                row[f"{dt}_{xy}"] = {"us": round(t * 1e6, 2), "gflops": round(2 * A.nnz / t / 1e9, 1),
                                     "speedup_vs_fp64": round(t64 / t, 2), "roofline": _roof(nb, t, pk)}
            S.free()
        res[f"bs{bs}"] = row
        M.free()
    _emit("bsr_scaled16_stencil27_64cubed_4dof", n=A.rows, nnz=A.nnz, variants=res)


def run_batch(bsp, dev, pk, up) -> None:
    """512 independent CSR matrices (half banded, half Zipf 2.2 rows), F64 and
    F32, 1 and 8 right-hand sides: one persistent graph launch vs one launch
    per matrix vs one cuSPARSE call per matrix."""
    import torch
    mats = bsp.gen_batch(512, SEED + 6)
    nnz = sum(int(m.rowptr[-1]) for m in mats)
    rows = sum(m.rows for m in mats)
    res = {}
    for dname, tdt, es in (("f64", torch.float64, 8), ("f32", torch.float32, 4)):
        base = [up(m.rowptr, m.colidx) + [torch.from_numpy(m.values).to(tdt).to(dev)] for m in mats]
        for nrhs in (1, 8):
            g = torch.Generator(device="cpu").manual_seed(nrhs)
            d = []
            for m, (rp, ci, va) in zip(mats, base):
                shp = (m.cols, nrhs) if nrhs > 1 else (m.cols,)
                xx = (torch.rand(shp, generator=g, dtype=torch.float64) * 2 - 1).to(tdt).to(dev)
                yy = torch.empty((m.rows, nrhs) if nrhs > 1 else (m.rows,), dtype=tdt, device=dev)
                d.append((rp, ci, va, xx, yy))
            P = bsp.BatchPlan(d, nrhs=nrhs, tune=1)
            tb = _timed(P.run, 50)
            ts = _timed(P.run_separate, 5)
            choice = {int(k): int(v) for k, v in zip(*np.unique(P.lanes(), return_counts=True))}
            n_sell = int((P.formats() == 1).sum())
            Pm = bsp.BatchPlan(d, nrhs=nrhs, tune=0)
            tm = _timed(Pm.run, 50)
            Pm.close()
            nb = nnz * (es + 4) + (rows + len(mats)) * 4 + 2 * rows * nrhs * es
            res[f"{dname}_rhs{nrhs}"] = {"batched_us": round(tb * 1e6, 1), "separate_us": round(ts * 1e6, 1),
                                         "speedup": round(ts / tb, 2), "gbs": round(nb / tb / 1e9, 1),
                                         "frac": round(nb / tb / 1e9 / pk, 4),
                                         "gflops": round(2 * nnz * nrhs / tb / 1e9, 1), "launches_batched": 1,
                                         "launches_separate": len(mats), "model_plan_us": round(tm * 1e6, 1),
                                         "lanes_chosen": choice, "sell32_matrices": n_sell}
            if nrhs == 1:
                fns = [_cusparse_spmv(rp, ci, va, xx, m.rows, m.cols) for m, (rp, ci, va, xx, _) in zip(mats, d)]
                res[f"{dname}_rhs1"]["cusparse_separate_us"] = round(_timed(lambda: [f() for f in fns], 5) * 1e6, 1)
            P.close()
    _emit("batch_512_banded_and_zipf2.2", matrices=len(mats), rows=rows, nnz=nnz, variants=res)


def run_cg_multi(bsp, up, dev) -> None:
    """FP64 CG to 1e-10 for 8 right-hand sides: one multi-RHS solve (the
    matrix read once per iteration for all columns) vs 8 single solves; the
    7-point Poisson 128^3 and the 4-dof block Laplacian 48^3 (28 entries per
    row) with Jacobi."""
    import torch
    for name, A, pc in (("cg_multi8_poisson3d_128", bsp.gen_poisson3d(128), "none"),
                        ("cg_multi8_block_laplace3d_48_4dof_jacobi", bsp.gen_block_laplace3d(48, 4, 10.0, SEED + 33),
                         "jacobi")):
        rp, ci, va = up(A.rowptr, A.colidx, A.values)
        g = torch.Generator(device="cpu").manual_seed(8)
        B = (torch.rand(A.rows, 8, generator=g, dtype=torch.float64) * 2 - 1).to(dev)
        S = bsp.CgSolver(rp, ci, va, mode="fp64", precond=pc, max_iters=50000)
        S.solve_multi(B)                                            # warm-up
        _, rel, rm = S.solve_multi(B)
        single = 0.0
        its = []
        for j in range(8):
            bj = B[:, j].contiguous()
            S.solve(bj)
            _, r1 = S.solve(bj)
            single += r1["seconds"]
            its.append(r1["iterations"])
        S.close()
        _emit(name, n=A.rows, nnz=A.nnz, k=8, precond=pc,
              multi={"ms": round(rm["seconds"] * 1e3, 3), "iterations": rm["iterations"],
                     "worst_rel_residual": float(rel.max()),
                     "gbs": round(rm["bytes_moved"] / rm["seconds"] / 1e9, 1)},
              eight_single={"ms": round(single * 1e3, 3), "iterations": its},
              speedup=round(single / rm["seconds"], 2))
        del rp, ci, va, B


def run_pcg(bsp, up) -> None:
    """CG to 1e-10 with no / Jacobi / block-Jacobi preconditioning, FP64 and
    mixed storage: a 4-dof block Laplacian L (x) S (64^3 nodes, cond(S) = 1e3)
    and a 7-point diffusion with 400x coefficient contrast (128^3).  The CPU
    line is the oracle's FP64 PCG (one thread) on the block Laplacian with
    block-Jacobi, the best method."""
    import time

    from oracle import pyoracle
    # FP16 storage of the block Laplacian (cond(A) ~ 1e6) is too coarse (the
    # solver says so and stops); its mixed line uses FP32 storage
    for name, A, pcs, modes in (("pcg_block_laplace3d_64_4dof_cond1e3",
                                 bsp.gen_block_laplace3d(64, 4, 1e3, SEED + 30),
                                 (("none", 4), ("jacobi", 4), ("block_jacobi", 4)), ("fp64", "f32")),
                                ("pcg_diffusion3d_128_contrast3", bsp.gen_diffusion3d(128, 3.0, SEED + 31),
                                 (("none", 4), ("jacobi", 4)), ("fp64", "f16"))):
        bh = bsp.gen_uniform(A.rows, SEED + 32)
        rp, ci, va, b = up(A.rowptr, A.colidx, A.values, bh)
        res = {}
        for pc, blk in pcs:
            for mode in modes:
                S = bsp.CgSolver(rp, ci, va, mode=mode, tol=1e-10, precond=pc, block=blk,
                                 max_iters=20000 if pc == "none" else 50000)
                S.solve(b, raise_on_stall=False)             # warm-up (captures the iteration graphs)
                _, best = S.solve(b, raise_on_stall=False)
                S.close()
                res[f"{pc}_{mode}"] = {"ms": round(best["seconds"] * 1e3, 3), "iterations": best["iterations"],
                                       "converged": bool(best["converged"]), "rel_residual": best["rel_residual"],
                                       "outer_steps": best["outer_steps"],
                                       "gbs": round(best["bytes_moved"] / best["seconds"] / 1e9, 1)}
        extra = {}
        if "block_jacobi" in dict(pcs):
            t0 = time.perf_counter()
            _, it = pyoracle.pcg(A.rowptr, A.colidx, A.values, bh, 4, 1e-10)
            t_cpu = time.perf_counter() - t0
            extra["cpu_baseline"] = {"value": round(t_cpu * 1e3, 1), "unit": "ms", "cores": 1, "kind": "port",
                                     "iterations": it, "sample": "oracle FP64 block-Jacobi PCG, full matrix"}
        ok = [k for k in res if res[k]["converged"]]
        best_key = min(ok, key=lambda k: res[k]["ms"]) if ok else None
        _emit(name, n=A.rows, nnz=A.nnz, variants=res, fastest=best_key,
              speedup_vs_unpreconditioned_fp64=(round(res["none_fp64"]["ms"] / res[best_key]["ms"], 2)
                                                if best_key and res["none_fp64"]["converged"] else None), **extra)
        del rp, ci, va, b


def run_reorder_similarity(bsp, dev, up) -> None:
    """The SMaT workload (524,288 rows, 8 dense 16x16 tiles per 16-row
    block, random block columns) with its rows shuffled: every tile then
    holds one row.  Row-similarity reordering (host, one-time) regroups the
    rows; SMaT tcgen05 SpMM at N = 128 on the shuffled and the reordered
    rows (whose product is the shuffled one with rows permuted), and the
    grouped CSR SpMM, the engine for scattered rows, on the shuffled rows."""
    import time

    import torch
    T = bsp.gen_random_bsr(32768, 16, 8, 1.0, 1.0, SEED + 5)
    S = bsp.permute_rows_csr_host(T, np.random.default_rng(SEED + 40).permutation(T.rows).astype(np.int32))
    del T
    t0 = time.perf_counter()
    perm = bsp.reorder_similarity_host(S.rowptr, S.colidx, S.cols)
    reorder_s = time.perf_counter() - t0
    R = bsp.permute_rows_csr_host(S, perm)
    N = 128
    choice, _ = bsp.choose_spmm_host(S, N)
    B = (torch.rand(S.cols, N, generator=torch.Generator().manual_seed(3)) * 2 - 1).half().to(dev)
    res, C = {}, {}
    for name, M in (("shuffled", S), ("reordered", R)):
        rp, ci, va = up(M.rowptr, M.colidx, M.values)
        Sm = bsp.SmatMatrix(rp, ci, va, rows=M.rows, cols=M.cols, dtype="f16")
        C[name] = Sm.spmm(B, path="tcgen05")
        t = _timed(lambda: Sm.spmm(B, C[name], path="tcgen05"), 10)
        res[name] = {"smat_tcgen05_ms": round(t * 1e3, 4), "tflops": round(2 * M.nnz * N / t / 1e12, 2),
                     "tile_fill": round(Sm.fill, 4)}
        if name == "shuffled":
            v16 = va.half()
            t = _timed(lambda: bsp.spmm_csr(rp, ci, v16, B), 5)
            res[name]["csr_grouped_ms"] = round(t * 1e3, 4)
        Sm.check()
        Sm.free()
        del rp, ci, va
    same = bool(torch.allclose(C["reordered"], C["shuffled"][torch.from_numpy(perm).long().to(dev)],
                               rtol=1e-5, atol=1e-5))
    _emit("reorder_similarity_shuffled_tiles_524k_N128", rows=S.rows, nnz=S.nnz, reorder_host_s=round(reorder_s, 3),
          variants=res, speedup_vs_shuffled_smat=round(res["shuffled"]["smat_tcgen05_ms"] /
                                                       res["reordered"]["smat_tcgen05_ms"], 2),
          speedup_vs_shuffled_best=round(min(res["shuffled"]["smat_tcgen05_ms"], res["shuffled"]["csr_grouped_ms"]) /
                                         res["reordered"]["smat_tcgen05_ms"], 2),
          product_rows_match=same,
          engine_choice={k: choice[k] for k in ("engine", "smat_path", "reorder", "est_seconds_smat_given",
                                                "est_seconds_smat_reordered", "est_seconds_csr")})


def run_mtx_read(bsp, dev) -> None:
    """File -> device CSR through the library vs scipy.io.mmread (the
    fast_matrix_market reader the reference's drivers use) + a stable
    (row, col) sort, the reference's conversion; median of 3 each."""
    import os
    import tempfile
    import time
    import warnings

    import scipy.io
    import torch
    A = bsp.gen_stencil27(32, 4, SEED + 20)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "stencil.mtx")
        bsp.write_mtx(path, A)
        mb = os.path.getsize(path) / 1e6

        def ours():
            f = bsp.MtxFile(path)
            t1 = time.perf_counter()
            out = f.csr(dev)
            torch.cuda.synchronize()
            f.close()
            return out, t1

        def theirs():
            with warnings.catch_warnings():
                warnings.simplefilter("ignore")
                m = scipy.io.mmread(path)
            o = np.lexsort((m.col, m.row))
            rp = np.zeros(m.shape[0] + 1, np.int64)
            np.add.at(rp, m.row.astype(np.int64) + 1, 1)
            return np.cumsum(rp), m.col[o], m.data[o]

        t_ours, t_parse, t_ref = [], [], []
        for _ in range(3):
            t0 = time.perf_counter()
            (rp, ci, va), t1 = ours()
            t2 = time.perf_counter()
            t_ours.append(t2 - t0)
            t_parse.append(t1 - t0)
            t0 = time.perf_counter()
            R = theirs()
            t_ref.append(time.perf_counter() - t0)
        same = (np.array_equal(rp.cpu().numpy(), R[0]) and np.array_equal(ci.cpu().numpy(), R[1])
                and np.array_equal(va.cpu().numpy().view(np.uint64), R[2].astype(np.float64).view(np.uint64)))
    to, tp, tr = (float(np.median(t)) for t in (t_ours, t_parse, t_ref))
    _emit("mtx_read_stencil27_32cubed_4dof", nnz=A.nnz, file_mb=round(mb, 1), threads=os.cpu_count(),
          ours={"file_to_device_csr_s": round(to, 4), "parse_s": round(tp, 4), "mb_per_s": round(mb / to, 1)},
          scipy_fmm_plus_sort={"file_to_host_csr_s": round(tr, 4), "mb_per_s": round(mb / tr, 1)},
          speedup=round(tr / to, 2), identical_csr=bool(same))


# ---------------------------------------------------------------------------
# --profile W: a few calls of one workload's kernels, for ncu captures (small
# enough to capture, inputs still larger than L2).  Prints one line.

def run_profile(args) -> None:
    import torch

    import benchsp_b200 as bsp
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    reps = max(1, min(args.steps, 5))

    def up(*arrs):
        return [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in arrs]

    w = args.profile
    if w == "dasp":   # power-law rows, Zipf 2.0 capped at 10k, n = 2^21 (190 MB of CSR)
        A = bsp.gen_powerlaw(1 << 21, 2.0, 10000, SEED + 13)
        rp, ci, va, x = up(A.rowptr, A.colidx, A.values, bsp.gen_uniform(A.cols, SEED + 14))
        D = bsp.csr2dasp(rp, ci, va, rows=A.rows, cols=A.cols)
        y = torch.empty(A.rows, dtype=torch.float64, device=dev)
        for _ in range(reps):
            D.spmv(x, y)
    elif w in ("cg_fp64", "cg_f16"):   # 7-point Poisson 128^3, 32 iterations, no graphs
        A = bsp.gen_poisson3d(128)
        rp, ci, va, b = up(A.rowptr, A.colidx, A.values, bsp.gen_uniform(A.rows, SEED + 3))
        S = bsp.CgSolver(rp, ci, va, mode=w[3:], max_iters=32, check_every=16, use_graphs=False)
        S.solve(b, raise_on_stall=False)
    elif w == "spmm":   # power-law graph 2^20, FP16, N = 128 (or --pn), planned (slab engine)
        A = bsp.gen_graph(1 << 20, 1.8, 32, SEED + 4)
        rp, ci, v64 = up(A.rowptr, A.colidx, A.values)
        v = v64.half()
        P = bsp.SpmmPlan(rp, ci, v, cols=A.cols, chunk=256)
        B = (torch.rand(A.cols, args.pn or 128, generator=torch.Generator().manual_seed(1)) * 2 - 1).half().to(dev)
        for _ in range(reps):
            P.spmm(B)
    elif w in ("smat_tc", "smat_mma", "smat_tc_w64", "smat_tc_w128", "smat_tcp", "smat_tcp_w64"):
        # dense 16x16 tiles, 8 per block-row, 524,288 rows, N = 256 (or --pn), FP16
        A = bsp.gen_random_bsr(32768, 16, 8, 1.0, 1.0, SEED + 5)
        rp, ci, va = up(A.rowptr, A.colidx, A.values)
        M = bsp.SmatMatrix(rp, ci, va, rows=A.rows, cols=A.cols, dtype="f16")
        B = (torch.rand(A.cols, args.pn or 256, generator=torch.Generator().manual_seed(1)) * 2 - 1).half().to(dev)
        path = {"smat_tc": "tcgen05", "smat_mma": "mma_sync", "smat_tc_w64": "tcgen05_w64",
                "smat_tc_w128": "tcgen05_w128", "smat_tcp": "tcgen05_persistent",
                "smat_tcp_w64": "tcgen05_persistent_w64"}[w]
        for _ in range(reps):
            M.spmm(B, path=path)
        M.check()
    elif w == "bsr_scaled":   # FP16 per-block-scaled 4x4 BSR, stencil 40^3 x 4 dof (> L2)
        A, xh = make_matrix(40)
        rp, ci, va, x = up(A.rowptr, A.colidx, A.values, xh)
        M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=4)
        S = M.scaled("f16")
        M.free()
        y = torch.empty(A.rows, dtype=torch.float64, device=dev)
        for _ in range(reps):
            S.spmv(x, y)
    elif w == "csr":   # CSR FP64 vector kernel, 2-D Laplacian 512x512 (21 MB; ncu replays cold-cache)
        A = bsp.gen_laplace2d(512, 512)
        rp, ci, va, x = up(A.rowptr, A.colidx, A.values, bsp.gen_uniform(A.cols, SEED + 10))
        y = torch.empty(A.rows, dtype=torch.float64, device=dev)
        for _ in range(reps):
            bsp.csr_spmv(rp, ci, va, x, y)
    elif w == "pcg_bj":   # block-Jacobi PCG, block Laplacian 48^3 x 4 dof (145 MB of CSR), 32 iterations
        A = bsp.gen_block_laplace3d(48, 4, 1e3, SEED + 30)
        rp, ci, va, b = up(A.rowptr, A.colidx, A.values, bsp.gen_uniform(A.rows, SEED + 32))
        S = bsp.CgSolver(rp, ci, va, mode="fp64", precond="block_jacobi", block=4, max_iters=32, check_every=16,
                         use_graphs=False)
        S.solve(b, raise_on_stall=False)
    elif w == "cg_multi":   # FP64 CG for 8 right-hand sides, 7-point Poisson 128^3 (~1 GB), 32 iterations
        A = bsp.gen_poisson3d(128)
        rp, ci, va = up(A.rowptr, A.colidx, A.values)
        g = torch.Generator(device="cpu").manual_seed(8)
        B = (torch.rand(A.rows, 8, generator=g, dtype=torch.float64) * 2 - 1).to(dev)
        S = bsp.CgSolver(rp, ci, va, mode="fp64", max_iters=32, check_every=16)
        S.solve_multi(B, raise_on_stall=False)
    elif w == "spmm_grouped":   # power-law graph 2^20, FP16, N = 128, grouped CSR engine
        A = bsp.gen_graph(1 << 20, 1.8, 32, SEED + 4)
        rp, ci, v64 = up(A.rowptr, A.colidx, A.values)
        v = v64.half()
        B = (torch.rand(A.cols, 128, generator=torch.Generator().manual_seed(1)) * 2 - 1).half().to(dev)
        C_out = torch.empty(A.rows, 128, dtype=torch.float32, device=dev)
        for _ in range(reps):
            bsp.spmm_csr(rp, ci, v, B, C_out)
    elif w in ("batch", "batch8"):   # the 512-matrix batch, FP64, one RHS (batch8: 8 right-hand sides)
        mats = bsp.gen_batch(512, SEED + 6)
        nrhs = 8 if w == "batch8" else 1
        d = []
        for m in mats:
            rp, ci, va = up(m.rowptr, m.colidx, m.values)
            shp = (m.cols, nrhs) if nrhs > 1 else (m.cols,)
            x = (torch.rand(shp, generator=torch.Generator().manual_seed(1), dtype=torch.float64) * 2 - 1).to(dev)
            d.append((rp, ci, va, x, torch.empty((m.rows, nrhs) if nrhs > 1 else (m.rows,), dtype=torch.float64,
                                                 device=dev)))
        P = bsp.BatchPlan(d, nrhs=nrhs, use_graph=False)
        for _ in range(reps):
            P.run()
    else:
        raise SystemExit(f"unknown profile workload {w}")
    torch.cuda.synchronize()
    print(json.dumps({"profile": w, "calls": reps}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cg", action="store_true", help="skip the CG figures in the headline line's extra")
    ap.add_argument("--suite", action="store_true", help="one JSON line per further workload (1 GPU)")
    ap.add_argument("--grid", type=int, default=GRID, help="stencil grid edge (64 = the benchmark config; "
                    "smaller values only for profiling captures)")
    ap.add_argument("--profile", choices=["dasp", "cg_fp64", "cg_f16", "spmm", "batch", "smat_tc", "smat_mma", "csr",
                                          "pcg_bj", "spmm_grouped", "cg_multi", "smat_tc_w64", "smat_tc_w128",
                                          "bsr_scaled", "smat_tcp", "smat_tcp_w64", "batch8"],
                    help="a few calls of one workload's kernels (for ncu captures)")
    ap.add_argument("--pn", type=int, default=0, help="columns of B for the SpMM profile workloads "
                    "(default 128 for spmm, 256 for the smat ones)")
    args = ap.parse_args()
    if args.profile:
        run_profile(args)
        return
    if args.suite:
        run_suite(args)
        return
    ws, rank, local = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
