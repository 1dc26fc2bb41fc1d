#!/usr/bin/env python3
"""Benchmark of the B200 tiled SpGEMM (FP64, 16x16 tiles).

Workload (N=1): C = A*A for the 27-point stencil on a 64^3 grid
(n = 262,144, nnz(A) = 6,859,000, FP64 values uniform(0.5, 1.5)), the largest
of the benchmark configurations whose product fits one GPU (the R-MAT scale-20
product, ~197 GB of C, does not).  A "step" is one product, steps 1-3 of the
tiled method including the allocation of C (the reference's timing window,
src/tilespgemm-cuda.h:2745-3124), with A resident in HBM as tiles.  L2 (126
MB) is flushed by a 512 MiB write before every timed step, outside the timed
events.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank computes its own product (independent replicas: the
product has no exchange step); value = products of all ranks / max rank time.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "rw-spgemm_b200"
METRIC = "SpGEMM GFLOP/s & HBM GB/s vs plain path; served jobs/s with p50/p99 latency"


def _load(name, path, pkg_dir=None):
    if name in sys.modules:
        return sys.modules[name]
    kw = {"submodule_search_locations": [str(pkg_dir)]} if pkg_dir else {}
    spec = importlib.util.spec_from_file_location(name, path, **kw)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(workload_key):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (profiles/k_step3_<workload>.md, line 'traffic_bytes_per_launch:')."""
    p = ROOT / "profiles" / f"k_step3_{workload_key}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return int(float(line.split(":", 1)[1].strip()))
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = Path("/tmp") / f"tsg_clocks_{os.getpid()}.csv"

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if not self.proc or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload_matrix(gen):
    return gen.stencil_27pt_3d(64, seed=0)


def compulsory_bytes(tA, tB, numC, nnzC):
    """Tiled A read + tiled B read + tiled C written (bytes)."""
    def tiled(tilem, T, nnz):
        return 4 * (tilem + 1) + 4 * T + 4 * (T + 1) + 16 * T + 32 * T + 9 * nnz
    a = tiled(tA.s.tilem, tA.numtile, tA.nnz)
    b = tiled(tB.s.tilem, tB.numtile, tB.nnz) + 4 * (tB.s.tilen + 1) + 8 * tB.numtile
    c = 4 * (tA.s.tilem + 1) + 8 * numC + 4 * (numC + 1) + 16 * numC + 32 * numC + 9 * nnzC
    return a + b + c


def step3_algorithmic_bytes(tA, tB, numC, nnzC):
    """Bytes the numeric kernel must move once: A and B tile data (Ptr, Col,
    Val, tile offsets and indices), C's structure (row/col, offsets, masks, Ptr)
    read, and C's Col + Val written."""
    def data(T, nnz):
        return 9 * nnz + 16 * T + 4 * (T + 1) + 4 * T
    a = data(tA.numtile, tA.nnz) + 4 * (tA.s.tilem + 1)
    b = data(tB.numtile, tB.nnz) + 4 * (tB.s.tilen + 1) + 8 * tB.numtile
    c = 8 * numC + 4 * (numC + 1) + 32 * numC + 16 * numC + 9 * nnzC
    return a + b + c


# ---------------------------------------------------------------------------
# CPU reference arm: the reference's own spgemm_cpu (serial, FP64) on a
# bounded row sample of the same workload.
# ---------------------------------------------------------------------------
def row_sample(mat, frac_den):
    m, n, rp, ci, v = mat
    rows = max(16, (m // frac_den) // 16 * 16)
    e = int(rp[rows])
    return rows, n, rp[:rows + 1].copy(), ci[:e].copy(), v[:e].copy()


def cpu_reference_step(oracle, sampleA, B_tiles):
    A_tiles = oracle.ref_csr2tile_row_major(sampleA)
    t0 = time.perf_counter()
    oracle.ref_spgemm_cpu(A_tiles, B_tiles)
    return time.perf_counter() - t0


def run_cpu_reference(args, gen, world, rank):
    if rank != 0:
        return None
    oracle = _load("tsg_oracle_py", ROOT / "oracle" / "oracle.py")
    mat = workload_matrix(gen)
    sample = row_sample(mat, 8)
    prods = int(oracle.count_products(sample, mat))
    kind = "reference" if oracle.ref_available() else "port"
    if kind == "reference":
        B_tiles = oracle.ref_csr2tile_col_major(mat)
        step = lambda: cpu_reference_step(oracle, sample, B_tiles)  # noqa: E731
        cores = 1
        what = "reference spgemm_cpu (src/spgemm-cpu.h:369, serial FP64, unpacked A bytes)"
    else:
        nthreads = os.cpu_count() or 1

        def step():
            t0 = time.perf_counter()
            oracle.gustavson(sample, mat, nthreads=nthreads)
            return time.perf_counter() - t0
        cores = nthreads
        what = "oracle port (element-level Gustavson, OpenMP)"
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    os.dup2(devnull, 1)  # the reference prints per call
    try:
        for _ in range(args.warmup):
            step()
        times = [step() for _ in range(args.steps)]
    finally:
        os.dup2(saved, 1)
        os.close(devnull)
    t = float(np.mean(times))
    gflops = 2.0 * prods / t / 1e9
    return {"value": gflops, "unit": "GFLOP/s", "cores": cores, "kind": kind,
            "sample": f"rows 0..{sample[0]} of the workload's A (1/8 of its rows) times the full A; "
                      f"{prods} products; {what}", "seconds_per_step": t}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, tsg, gen, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    mat = workload_matrix(gen)
    m, n, rp, ci, v = mat
    stream = torch.cuda.current_stream(dev)
    ctx = tsg.Context(local, stream=stream.cuda_stream)
    ctx.set_schedule(args.sched, args.seg, args.cap)
    d_rp = torch.from_numpy(rp).to(dev)
    d_ci = torch.from_numpy(ci).to(dev)
    d_v = torch.from_numpy(v).to(dev)
    A = tsg.csr_to_tiled(ctx, m, n, d_rp, d_ci, d_v, tsg.TSG_TILED_CSC_VIEW)  # serves as A and B
    prods = tsg.count_products(ctx, d_ci, d_rp)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def one_step():
        C, info = tsg.spgemm(ctx, A, A)
        return C, info

    for _ in range(max(args.warmup, 1)):
        C, info = one_step()
        C.free()
    torch.cuda.synchronize()
    ctx.set_timing(True)
    step_ms, s3_ms, infos = [], [], []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            C, info = one_step()
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            s3_ms.append(info["ms_step3"])
            infos.append(info)
            numC, nnzC = info["numtile_C"], info["nnz_C"]
            C.free()
        torch.cuda.synchronize()
    launches = ctx.launches() - launches0
    if dist:
        dist.barrier()
    ctx.set_timing(False)
    total_ms = float(np.sum(step_ms))
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = 2.0 * prods * world / (ms_per_step * 1e-3) / 1e9

    # roofline of the dominant kernel (numeric step)
    peak, peak_src = measured_peak_hbm()
    s3 = float(np.mean(s3_ms))
    alg3 = step3_algorithmic_bytes(A, A, numC, nnzC)
    achieved = alg3 / (s3 * 1e-3) / 1e9
    comp = compulsory_bytes(A, A, numC, nnzC)

    # end to end through the C ABI with host buffers (pinned inputs)
    e2e_t, h2d, d2h = float("nan"), 0, 0
    if not args.no_e2e:
        pin = lambda x: torch.from_numpy(x).pin_memory().numpy()  # noqa: E731
        hmat = (m, n, pin(rp), pin(ci), pin(v))
        tsg.spgemm_csr_host(ctx, hmat)
        e2e_ms = []
        for _ in range(max(2, min(args.steps, 5))):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            Cc, _ = tsg.spgemm_csr_host(ctx, hmat)
            torch.cuda.synchronize()
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
        e2e_t = float(np.mean(e2e_ms))
        h2d = rp.nbytes + ci.nbytes + v.nbytes
        d2h = Cc[2].nbytes + Cc[3].nbytes + Cc[4].nbytes

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_reference(argparse.Namespace(warmup=0, steps=1), gen, 1, 0)
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "C = A*A, 27-point stencil on a 64^3 grid (n=262,144, nnz=6,859,000, FP64 "
                               "uniform(0.5,1.5)), natural order, 16x16 tiles",
                   "products": prods, "tiles_A": A.numtile, "tiles_C": numC, "nnz_C": nnzC,
                   "window": "steps 1-3 incl. C allocation (reference tilespgemm window)",
                   "schedule": f"{args.sched} seg={args.seg} cap={args.cap}",
                   "l2": "512 MiB write before every timed step, outside the timed events",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "hbm_gbs": round(comp / (ms_per_step * 1e-3) / 1e9, 2),
        "hbm_frac": round(comp / (ms_per_step * 1e-3) / 1e9 / peak, 4),
        "compulsory_bytes": comp,
        "step_ms": {k: round(float(np.mean([i[k] for i in infos])), 4) for k in ("ms_step1", "ms_step2", "ms_step3")},
        "roofline": {"bound": "hbm", "kernel": "k_step3 (numeric)", "achieved": round(achieved, 2),
                     "peak": peak, "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "algorithmic_bytes": alg3, "traffic": profiled_traffic("stencil27_64")},
        "e2e": {"value": round(2.0 * prods / (e2e_t * 1e-3) / 1e9, 3), "unit": "GFLOP/s", "ms": round(e2e_t, 3),
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "path": "tsg_spgemm_csr_host (host CSR in -> host CSR out, pinned inputs)"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if cpu:
        out["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--sched", default="rows", choices=["rows", "tiles"])
    ap.add_argument("--seg", type=int, default=16)
    ap.add_argument("--cap", type=int, default=1024)
    args = ap.parse_args()
    world, rank, local = dist_setup()
    tsg = _load("rw_spgemm_b200", PKG_DIR / "__init__.py", PKG_DIR)
    gen = _load("rw_spgemm_b200.generators", PKG_DIR / "generators.py")
    if args.impl == "reference":
        res = run_cpu_reference(args, gen, world, rank)
        if rank == 0:
            line = {"metric": METRIC, "impl": "reference", "value": round(res["value"], 4), "unit": "GFLOP/s",
                    "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                    "ms_per_step": round(res["seconds_per_step"] * 1e3, 3), "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                    "config": {"workload": "C = A*A, 27-point stencil on a 64^3 grid (n=262,144), row sample",
                               "sample": res["sample"]},
                    "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
                    "e2e": {"value": round(res["value"], 4), "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        return
    run_ours(args, tsg, gen, world, rank, local)


if __name__ == "__main__":
    main()
