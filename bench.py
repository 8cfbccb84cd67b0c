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

def cpu_reference(A, x, max_seconds: float = 12.0, min_reps: int = 2) -> dict:
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
    bounds = np.linspace(0, A.rows, cores + 1).astype(np.int64)

    def run(t):
        r0, r1 = int(bounds[t]), int(bounds[t + 1])
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

    times = []
    t_start = time.perf_counter()
    while len(times) < min_reps or (time.perf_counter() - t_start < max_seconds and len(times) < 50):
        ths = [threading.Thread(target=run, args=(t,)) for t in range(cores)]
        t0 = time.perf_counter()
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return {"gflops": 2.0 * A.nnz / t / 1e9, "cores": cores, "kind": kind, "reps": len(times),
            "seconds_per_spmv": t, "y": y}


def make_matrix(grid: int = GRID):
    import benchsp_b200 as bsp
    A = bsp.gen_stencil27(grid, DOF, SEED)
    x = bsp.gen_uniform(A.cols, SEED + 1)
    return A, x


def run_reference(args, ws, rank):
    if rank != 0:
        return
    A, x = make_matrix(args.grid)
    ref = cpu_reference(A, x, max_seconds=max(2.0, min(60.0, 0.6 * args.steps)), min_reps=max(1, args.warmup))
    v = ref["gflops"]
    line = {
        "metric": METRIC, "value": round(v, 3), "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": ref["reps"],
        "warmup": args.warmup, "ms_per_step": round(ref["seconds_per_spmv"] * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "n": A.rows, "nnz": A.nnz, "block": "4x4",
                   "l2": "working set > L2"},
        "impl": "reference",
        "cpu_baseline": {"value": round(v, 3), "unit": "GFLOP/s", "cores": ref["cores"], "kind": ref["kind"],
                         "sample": f"full matrix, median of {ref['reps']} SpMVs, rows split over "
                                   f"{ref['cores']} threads"},
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
    ms = ev0.elapsed_time(ev1)
    if ws > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
        torch.distributed.barrier()
    ms_step = ms / args.steps
    value = ws * flops * args.steps / (ms / 1e3) / 1e9

    # e2e through the host-buffer C-ABI call: H2D x, SpMV, D2H y per step
    xh = torch.from_numpy(x_h).pin_memory()
    yh = torch.empty(A.rows, dtype=torch.float64).pin_memory()
    xh_np, yh_np = xh.numpy(), yh.numpy()
    e2e_steps = max(3, min(args.steps, 200))
    for _ in range(3):
        M.spmv_host(xh_np, yh_np)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        M.spmv_host(xh_np, yh_np)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if ws > 1:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = ws * flops * e2e_steps / (e2e_ms / 1e3) / 1e9

    # correctness of the benchmarked result (cheap, outside the timed region)
    y_np = y.cpu().numpy()
    ok = bool(np.allclose(y_np, yh_np, rtol=0, atol=0))

    if rank != 0:
        return
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
        "config": {"workload": WORKLOAD if args.grid == GRID else f"bsr4_fp64_spmv_stencil27_{args.grid}cubed_4dof",
                   "n": A.rows, "nnz": A.nnz, "blocks": M.blc_num, "block": "4x4",
                   "parallelism": f"replicas{ws}", "l2": "inputs larger than L2 (923 MB working set)",
                   "kernel": "bsr_ffma_kernel<4,16,1>"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / pk["hbm_gbs"], 4), "traffic": traffic,
                     "peak_src": pk["src"], "algorithmic_bytes_per_launch": algo_bytes},
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_value, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 8 * A.cols,
                "d2h_bytes_per_step": 8 * A.rows, "steps": e2e_steps},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "extra": {"csr2bsr_seconds": round(convert_s, 4), "gbs": round(achieved, 1),
                  "e2e_matches_device_result": ok},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", type=int, default=GRID, help="stencil grid edge (64 = the benchmark config; "
                    "smaller values only for profiling captures)")
    args = ap.parse_args()
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
