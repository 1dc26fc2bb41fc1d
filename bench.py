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

Under torchrun each rank computes its own stencil product (independent
replicas: the product has no exchange step); value = products of all ranks /
max rank time.  The R-MAT scale-20 products (C ~ 9.7e9 nonzeros) run as one
row-partitioned product over the ranks instead ("rmat20_sharded"): each rank
owns a range of A's tile rows cut by predicted products, holds all of B, and
computes its range in row blocks; one all-gather of (rows, nnz) places the
pieces.
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


def profiled_traffic(workload_key, sched):
    """Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of
    the numeric kernel from the committed ncu summary
    (profiles/numeric_step_<workload>.md, line 'traffic_bytes_per_launch[<sched>]:')."""
    p = ROOT / "profiles" / f"numeric_step_{workload_key}.md"
    if not p.exists():
        return None
    tag = f"traffic_bytes_per_launch[{sched}]:"
    for line in p.read_text().splitlines():
        if line.strip().startswith(tag):
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
        self.q = q
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "10"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            # the timed region can be a few ms: start it only once sampling runs
            t0 = time.time()
            while time.time() - t0 < 5.0 and self.path.stat().st_size == 0 and self.proc.poll() is None:
                time.sleep(0.01)
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
            # and one reading right at the end of the region
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=20)
                with open(self.path, "a") as fh:
                    fh.write(out.stdout)
            except (OSError, subprocess.SubprocessError):
                pass

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


def max_over_ranks(value, dist=None, device=None):
    """The largest of every rank's value (the job's time is its slowest
    rank's); the value itself without a process group."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist=None, device=None):
    """The sum of every rank's value; the value itself without a process
    group."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def replica_gflops(products_per_rank, world, ms_per_step):
    """Whole-job GFLOP/s of `world` independent replicas, each computing
    products_per_rank scalar products per step (2 flops each)."""
    return 2.0 * products_per_rank * world / (ms_per_step * 1e-3) / 1e9


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
# CPU reference arm: the reference's own CPU SpGEMM codes on a bounded row
# sample of the same workload -- spgemm_cpu (serial, FP64 numeric, the
# tiled method) and spgemm_spa (OpenMP over rows on all host threads, C's
# structure by a bitmap accumulator) -- the faster of the two is the baseline.
# ---------------------------------------------------------------------------
def host_cpu():
    """(logical CPUs usable here, CPU model)."""
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count() or 1
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return usable, model


def time_spa_step(oracle, sample, mat):
    t0 = time.perf_counter()
    oracle.ref_spgemm_spa(sample, mat)
    return time.perf_counter() - t0


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
    usable, model = host_cpu()
    spa = None
    if kind == "reference":
        B_tiles = oracle.ref_csr2tile_col_major(mat)
        step = lambda: cpu_reference_step(oracle, sample, B_tiles)  # noqa: E731
        cores = 1
        what = "reference spgemm_cpu (src/spgemm-cpu.h:369, serial FP64, unpacked A bytes)"
        omp = int(oracle.rlib().ref_omp_max_threads())
        time_spa_step(oracle, sample, mat)  # warm-up (thread pool, pages)
        ts = [time_spa_step(oracle, sample, mat) for _ in range(max(1, args.steps))]
        spa = {"seconds_per_step": float(np.mean(ts)), "threads": omp,
               "gflops_equiv": 2.0 * prods / float(np.mean(ts)) / 1e9,
               "what": "reference spgemm_spa (src/spgemm_serialref_spa_new.h:7), both passes (row counts, "
                       "columns), OpenMP on %d threads; structure only, no values" % omp}
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
    out = {"value": gflops, "unit": "GFLOP/s", "cores": cores, "kind": kind,
           "sample": f"rows 0..{sample[0]} of the workload's A (1/8 of its rows) times the full A; "
                     f"{prods} products; {what}", "seconds_per_step": t,
           "host": {"nproc": usable, "cpu_model": model}}
    if spa:
        out["spgemm_cpu_serial"] = {"gflops": round(gflops, 4), "seconds_per_step": round(t, 4)}
        out["spgemm_spa_all_cores"] = {"gflops_equiv": round(spa["gflops_equiv"], 4),
                                       "seconds_per_step": round(spa["seconds_per_step"], 4),
                                       "omp_threads": spa["threads"], "what": spa["what"]}
        out["host"]["omp_max_threads"] = spa["threads"]
        if spa["gflops_equiv"] > gflops:
            # the faster reference code is the baseline (rate: 2 x scalar products / s)
            out.update(value=spa["gflops_equiv"], cores=spa["threads"], seconds_per_step=spa["seconds_per_step"],
                       sample=f"rows 0..{sample[0]} of the workload's A (1/8 of its rows) times the full A; "
                              f"{prods} products; {spa['what']}; value = 2 x products / s (GFLOP/s-equivalent), "
                              f"faster than the serial numeric spgemm_cpu ({gflops:.4f} GFLOP/s)")
    return out


# ---------------------------------------------------------------------------
# batched (512 uneven products in one persistent, graph-captured launch) vs
# the plain one-product-at-a-time path on the same GPU
# ---------------------------------------------------------------------------
def run_batched(args, tsg, gen, ctx, steps):
    import torch
    at = _load("rw_spgemm_b200.autotune", PKG_DIR / "autotune.py")
    mats = gen.batched_products(args.batch_count, seed=0)
    classes = gen.batched_product_classes(args.batch_count, seed=0)
    pairs = [(tsg.csr_host_to_tiled(ctx, a, tsg.TSG_TILED_CSC_VIEW), tsg.csr_host_to_tiled(ctx, b, tsg.TSG_TILED_CSC_VIEW))
             for a, b in mats]
    prods_each = [tsg.product_bounds(ctx, A, B)[0] for A, B in pairs]
    total_products = sum(prods_each)
    del mats
    tuner = at.Autotuner()
    choice = tuner.tune_batch(ctx, pairs, reps=1, use_cache=False)
    tune_ms = at.summarize(tuner.last_timings)
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(sub):
        """(ms per run of a graph-captured batch over sub, batch) -- batch
        left open, its last run finished."""
        b = at.make_batch(ctx, sub, choice, graph=True)
        b.run()
        b.sync()
        ctx.synchronize()
        ev[0].record(stream)
        for _ in range(steps):
            b.run()
        ev[1].record(stream)
        ev[1].synchronize()
        return ev[0].elapsed_time(ev[1]) / steps, b

    ms_batched, batch = timed(pairs)
    tiles, nnz = batch.sync()
    info = batch.info()
    phases = batch.phase_ms()
    batch.close()
    # the same batch split by product class, each class a batch of its own
    per_class = {}
    for cl in sorted(set(classes)):
        idx = [i for i, c in enumerate(classes) if c == cl]
        ms_c, b = timed([pairs[i] for i in idx])
        b.sync()
        ph = b.phase_ms()
        b.close()
        pc = sum(prods_each[i] for i in idx)
        per_class[cl] = {"products": int(pc), "count": len(idx), "ms": round(ms_c, 3),
                         "gflops": round(2.0 * pc / (ms_c * 1e-3) / 1e9, 2),
                         "phase_ms": ph}
    # plain path: one tsg_spgemm per product (its own launches, read-backs and allocations)
    ctx.set_schedule(*at.normalize(choice))
    for A, B in pairs[:8]:
        C, _ = tsg.spgemm(ctx, A, B)
        C.free()
    ctx.synchronize()
    ev[0].record(stream)
    for _ in range(max(1, steps // 2)):
        for A, B in pairs:
            C, _ = tsg.spgemm(ctx, A, B)
            C.free()
    ev[1].record(stream)
    ev[1].synchronize()
    ms_plain = ev[0].elapsed_time(ev[1]) / max(1, steps // 2)
    for A, B in pairs:
        A.free()
        B.free()
    gf_b = 2.0 * total_products / (ms_batched * 1e-3) / 1e9
    gf_p = 2.0 * total_products / (ms_plain * 1e-3) / 1e9
    return {"workload": f"{len(pairs)} independent FP64 products C_i = A_i*B_i, n_i log-uniform in [1024, 65536], "
                        "A_i/B_i banded (half-bandwidth 8-64) or random Poisson(8) per row, values U(-1,1)",
            "products": int(total_products), "C_tiles": int(tiles), "C_nnz": int(nnz),
            "gflops_batched": round(gf_b, 2), "gflops_plain": round(gf_p, 2), "speedup_vs_plain": round(gf_b / gf_p, 3),
            "ms_batched": round(ms_batched, 3), "ms_plain": round(ms_plain, 3),
            "phase_ms": phases, "per_class": per_class,
            "schedule": at.label(choice), "autotune_ms": tune_ms, "graph": info["graph"], "grid": info["grid"],
            "arena_gb": round(info["arena_bytes"] / 1e9, 3)}


# ---------------------------------------------------------------------------
# served: Poisson arrivals into the continuous-batching server
# ---------------------------------------------------------------------------
def _served_stream(srv, jobs, rate, rng):
    """Submits jobs with Poisson arrivals at `rate` jobs/s; returns the
    server's statistics and the wall time of the stream."""
    srv.done.clear()
    srv.batches = 0
    srv.host_s = dict.fromkeys(srv.host_s, 0.0)
    gaps = rng.exponential(1.0 / rate, len(jobs))
    futs = []
    t0 = time.perf_counter()
    t_next = t0
    for (kind, a, b, _), g in zip(jobs, gaps):
        t_next += g
        while True:
            now = time.perf_counter()
            if now >= t_next:
                break
            time.sleep(min(t_next - now, 0.0005))
        futs.append(srv.submit(kind, a, b))
    for f in futs:
        f.result(timeout=600)
    return srv.stats(), time.perf_counter() - t0


def run_served(args, tsg, gen, device, deliver="device", n_jobs=None, half_capacity=True):
    """deliver="device": results handed over as device tensors (the GPU
    service alone); "host": as numpy arrays in page-locked memory (every
    result crosses the bus)."""
    srv_mod = _load("rw_spgemm_b200.serve", PKG_DIR / "serve.py")
    pool = gen.served_pool()
    srv = srv_mod.SpGEMMServer(device, mem_cap=40 << 30, slots=2, max_batch=64, schedule=args.served_schedule,
                               deliver=deliver)
    for key, m in pool.items():
        srv.register(key, m)
    rng = np.random.default_rng(1)
    jobs = []
    for kind, a, b in gen.served_jobs(pool, n_jobs or args.served_jobs, seed=1):
        B = gen.transpose(pool[a]) if kind == "AAT" else pool[b]
        jobs.append((kind, a, b, gen.products(pool[a], B)))
    # warm the operand cache, the kernels and the tuned schedules with a pass
    # over the first jobs
    srv.start()
    for f in [srv.submit(k, a, b) for k, a, b, _ in jobs[:256]]:
        f.result(timeout=600)
    st, wall = _served_stream(srv, jobs, args.served_rate, rng)
    prods = sum(j[3] for j in jobs)
    out = {"workload": "Poisson arrivals at %d jobs/s; mix 85%% small batched-generator products (n 1k-16k), 10%% "
                       "R-MAT scale 14, 4%% scale 15, 1%% scale 16 (edge factor 8/16); 50%% A*B, 50%% A*A^T"
                       % args.served_rate,
           "jobs": st["jobs"], "jobs_per_s": round(st["jobs_per_s"], 1), "p50_ms": round(st["p50_ms"], 3),
           "p99_ms": round(st["p99_ms"], 3), "gflops": round(2.0 * prods / wall / 1e9, 2),
           "batches": st["batches"], "mean_batch": round(st["mean_batch"], 2), "rejected": st["rejected"],
           "operand_cache": st["operand_cache"], "mem_cap_gb": 40, "deliver": deliver,
           "dispatcher_s": dict(st["dispatcher_s"], wall=round(wall, 3)),
           "schedule": st["tuned"] if args.served_schedule == "auto" else "-".join(map(str, args.served_schedule))}
    if not half_capacity:
        srv.close()
        return out
    # the same mix below saturation: half the throughput the stream above reached
    rate2 = max(1.0, 0.5 * st["jobs_per_s"])
    sub = jobs[:max(100, min(len(jobs), int(rate2 * 10)))]
    st2, wall2 = _served_stream(srv, sub, rate2, rng)
    out["at_half_capacity"] = {"rate_jobs_per_s": round(rate2, 1), "jobs": st2["jobs"],
                               "jobs_per_s": round(st2["jobs_per_s"], 1), "p50_ms": round(st2["p50_ms"], 3),
                               "p99_ms": round(st2["p99_ms"], 3)}
    srv.close()
    return out


def run_served_plain(args, tsg, gen, ctx, n_jobs=None):
    """The served job stream run on the plain path instead: one tsg_spgemm
    per job (its own launches, host read-backs and allocations) and its
    conversion to device CSR, jobs back to back with operands resident --
    the plain path's best throughput on the same mix (no arrival gaps)."""
    import torch
    pool = gen.served_pool()
    jobs = gen.served_jobs(pool, n_jobs or args.served_jobs, seed=1)
    tiles, prods = {}, 0

    def operand(key, mat):
        if key not in tiles:
            tiles[key] = tsg.csr_host_to_tiled(ctx, mat, tsg.TSG_TILED_CSC_VIEW)
        return tiles[key]

    work = []
    for kind, a, b in jobs:
        Bkey = (a, "T") if kind == "AAT" else b
        Bm = gen.transpose(pool[a]) if kind == "AAT" and Bkey not in tiles else pool.get(b)
        A, B = operand(a, pool[a]), operand(Bkey, Bm)
        prods += tsg.product_bounds(ctx, A, B)[0]
        work.append((A, B))

    def one(A, B):
        C, _ = tsg.spgemm(ctx, A, B)
        out = tsg.tiled_to_csr(ctx, C)
        C.free()
        return out

    for A, B in work[:64]:
        one(A, B)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for A, B in work:
        one(A, B)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    for t in tiles.values():
        t.free()
    return {"what": "same job mix, one tsg_spgemm + tsg_tiled_to_csr per job, back to back, operands resident, "
                    "results left on the device", "jobs": len(work), "jobs_per_s": round(len(work) / wall, 1),
            "ms_per_job": round(wall * 1e3 / len(work), 3), "gflops": round(2.0 * prods / wall / 1e9, 2)}


# ---------------------------------------------------------------------------
# learned selector: trained on method-generated timings, measured against exhaustive
# search on held-out matrices
# ---------------------------------------------------------------------------
def run_selector(args, tsg, gen, ctx):
    sel = _load("rw_spgemm_b200.selector", PKG_DIR / "selector.py")
    n_mat = max(10, args.selector_samples // len(sel.CONFIGS))
    mats = sel.training_matrices(gen, n_mat, seed=21)
    t0 = time.perf_counter()
    data = [sel.time_configs(ctx, m, repeats=2) for m in mats]
    collect_s = time.perf_counter() - t0
    feats = np.stack([d[0] for d in data])
    times = np.stack([d[1] for d in data])
    order_ms = np.array([[d[2][o] for o in sel.ORDERINGS] for d in data])
    n_tr = int(0.8 * n_mat)
    net = sel.MLP(ctx, seed=3)
    t0 = time.perf_counter()
    losses = net.fit(feats[:n_tr], times[:n_tr], epochs=300, lr=2e-3)
    train_s = time.perf_counter() - t0
    te = slice(n_tr, n_mat)
    picks = np.argmin(net.predict(feats[te]), axis=1)
    fixed_best = int(np.argmin(np.log(times[:n_tr]).mean(0)))
    res = {
        "timing_samples": int(times.size), "matrices": n_mat, "train": n_tr, "held_out": n_mat - n_tr,
        "configs": [f"{o}/{a[0]}-{a[1]}-{a[2]}" for o, a in sel.CONFIGS],
        "regret_model": sel.regret(times[te], picks),
        "regret_without_model": sel.regret(times[te], np.zeros(n_mat - n_tr, dtype=int)),
        "regret_best_fixed": sel.regret(times[te], np.full(n_mat - n_tr, fixed_best)),
        "best_fixed_config": res_name(sel, fixed_best),
        "final_train_loss": round(float(losses[-1]), 5), "collect_s": round(collect_s, 1),
        "train_s": round(train_s, 2), "mean_ordering_ms": {o: round(float(order_ms[:, k].mean()), 3)
                                                           for k, o in enumerate(sel.ORDERINGS)},
        "within_10pct_of_exhaustive": bool(sel.regret(times[te], picks)[0] <= 0.10),
    }
    net.close()
    return res


def run_orderings(args, tsg, gen, ctx, reps=3):
    """27-point stencil on a 64^3 grid after a seeded random symmetric
    permutation; every GPU ordering is applied (permutation + CSR permute timed
    on the device), then C = A*A (steps 1-3, min of reps): tile count of C and
    run time per ordering."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    base = gen.stencil_27pt_3d(64, seed=0)
    mat = gen.permute_symmetric(base, gen.random_symmetric_permutation(base[0], 7))
    m, n, rp, ci, v = mat
    d_rp, d_ci, d_v = (torch.from_numpy(x).to(dev) for x in (rp, ci, v))
    prods = tsg.count_products(ctx, d_ci, d_rp)
    out = {"workload": "27-point stencil 64^3 (n=262,144), seeded random symmetric permutation, then each ordering; "
                       "C = A*A", "products": int(prods), "per_ordering": {}}
    ctx.set_timing(True)
    for name in ["original", "rcm", "degree", "gray", "random", "tasa"]:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best_order = float("inf")
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e0.record()
            if name == "tasa":
                # the tile-aware planner on the symmetric matrix (host plan:
                # one order for every axis), timed by the host clock
                plan = tsg.build_reorder_plan("AA", "tasa", mat, symmetric=True)
                perm = torch.from_numpy(np.ascontiguousarray(plan["row_perm"], np.int32)).to(dev)
            else:
                perm = tsg.order(ctx, name, m, n, d_rp, d_ci, seed=1)
            inv = torch.empty_like(perm)
            inv[perm.long()] = torch.arange(m, dtype=torch.int32, device=dev)
            prp, pci, pv = tsg.permute_csr(ctx, m, n, d_rp, d_ci, d_v, perm, inv)
            e1.record()
            e1.synchronize()
            took = (time.perf_counter() - t0) * 1e3 if name == "tasa" else e0.elapsed_time(e1)
            best_order = min(best_order, took)
        T = tsg.csr_to_tiled(ctx, m, n, prp, pci, pv, tsg.TSG_TILED_CSC_VIEW)
        best, info = float("inf"), None
        for _ in range(reps):
            C, inf = tsg.spgemm(ctx, T, T)
            if inf["ms_total"] < best:
                best, info = inf["ms_total"], inf
            C.free()
        if name == "tasa":
            out["tasa_plan"] = {"mode": plan["mode"], "risk_reason": plan["risk_reason"],
                                "window": plan["local_refine_window"]}
        out["per_ordering"][name] = {"ordering_ms": round(best_order, 3), "tiles_A": int(T.numtile),
                                     "tiles_C": int(info["numtile_C"]), "nnz_C": int(info["nnz_C"]),
                                     "ms_steps_1_3": round(best, 4),
                                     "gflops": round(2.0 * prods / (best * 1e-3) / 1e9, 2)}
        T.free()
        del prp, pci, pv
    ctx.set_timing(False)
    return out


def run_hyper(args, tsg, gen, ctx, reps=3):
    """The largest random product of the batched configuration: A and B
    65,536 x 65,536 with Poisson(8) nonzeros per row, C = A*B.  Step 1 lists
    nearly every tile column of each C tile row (16.4 M C tiles for 4.2 M
    values), so steps 2 and 3 run the hypersparse whole-row path.  Steps 1-3
    (min of reps, CUDA events)."""
    A = gen.random_poisson(65536, None, 8.0, seed=7)
    B = gen.random_poisson(65536, None, 8.0, seed=8)
    TA = tsg.csr_host_to_tiled(ctx, A, tsg.TSG_TILED_PACKED_COL)
    TB = tsg.csr_host_to_tiled(ctx, B, tsg.TSG_TILED_CSC_VIEW)
    prods = tsg.product_bounds(ctx, TA, TB)[0]
    ctx.set_timing(True)
    best, info = float("inf"), None
    for _ in range(reps):
        C, inf = tsg.spgemm(ctx, TA, TB)
        if inf["ms_total"] < best:
            best, info = inf["ms_total"], inf
        C.free()
    ctx.set_timing(False)
    TA.free()
    TB.free()
    return {"workload": "C = A*B, A and B 65,536 x 65,536 random with Poisson(8) nonzeros per row, FP64 U(-1,1)",
            "products": int(prods), "tiles_C": int(info["numtile_C"]), "nnz_C": int(info["nnz_C"]),
            "step_ms": {k: round(info[k], 4) for k in ("ms_step1", "ms_step2", "ms_step3")},
            "ms_steps_1_3": round(best, 4), "gflops": round(2.0 * prods / (best * 1e-3) / 1e9, 2)}


def run_rmat16(args, tsg, gen, ctx, reps=3):
    """One R-MAT product small enough to hold whole: scale 16, edge factor 16,
    C = A*A (the kind of work of one scale-20 row block: hub rows, C tile
    rows thousands of tiles wide with few values per tile).  Steps 1-3, min
    of reps, CUDA events."""
    A = gen.rmat(16, 16, seed=1)
    TA = tsg.csr_host_to_tiled(ctx, A, tsg.TSG_TILED_PACKED_COL)
    TB = tsg.csr_host_to_tiled(ctx, A, tsg.TSG_TILED_CSC_VIEW)
    prods = tsg.product_bounds(ctx, TA, TB)[0]
    ctx.set_timing(True)
    best = None
    for _ in range(reps):
        C, info = tsg.spgemm(ctx, TA, TB)
        C.free()
        if best is None or info["ms_total"] < best["ms_total"]:
            best = info
    ctx.set_timing(False)
    TA.free()
    TB.free()
    return {"workload": "R-MAT scale 16, edge factor 16 (n=65,536), C = A*A, FP64 U(-1,1)", "products": int(prods),
            "tiles_C": int(best["numtile_C"]), "nnz_C": int(best["nnz_C"]),
            "step_ms": {k: round(best[k], 3) for k in ("ms_step1", "ms_step2", "ms_step3")},
            "ms_steps_1_3": round(best["ms_total"], 3), "gflops": round(2.0 * prods / (best["ms_total"] * 1e-3) / 1e9, 2),
            "numeric_kernel": best["step3_name"]}


def run_rmat20(args, tsg, gen, ctx, budget=1.5e9, rank=0, world=1, dist=None, device=None):
    """R-MAT scale 20 (edge factor 16, a,b,c,d = .57,.19,.19,.05, duplicates
    merged, values U(-1,1)): C = A*A and C = A*A^T.  C (~9.7e9 nonzeros) does
    not fit one GPU, so A goes in blocks of tile rows holding at most `budget`
    scalar products each; every block is converted, multiplied (steps 1-3 on
    the resident B) and its C freed, after one untimed product of the
    largest block (the memory pool warmed).  With world > 1 the product is
    row-partitioned: this rank takes its tile-row range (shard.plan) and the
    time is the slowest rank's.  GFLOP/s over the steps-1-3 time of all
    blocks; wall time includes the block conversions; hbm_frac = compulsory
    tile bytes of every block (A block and B read, C written) / time / the
    measured copy bandwidth."""
    import torch
    blocks_mod = _load("rw_spgemm_b200.blocks", PKG_DIR / "blocks.py")
    shard = _load("rw_spgemm_b200.shard", PKG_DIR / "shard.py")
    peak, _ = measured_peak_hbm()
    A = gen.rmat(20, 16, seed=1)
    m, n, rp, ci, v = A
    out = {"workload": "R-MAT scale 20, edge factor 16 (n=1,048,576), FP64 U(-1,1); A in row blocks of <= %.1e "
                       "products" % budget}
    if world > 1:
        out["partition"] = (f"{world} ranks, consecutive tile-row ranges of A cut by predicted products, B "
                            "replicated per rank; time = slowest rank")
    for label, B in (("A*A", A), ("A*A^T", gen.transpose(A))):
        TB = tsg.csr_host_to_tiled(ctx, B, tsg.TSG_TILED_CSC_VIEW)
        tileprod, ranges = shard.plan(A, B, world)
        r0, r1 = ranges[rank]
        blocks = [(r0 + b0, r0 + b1) for b0, b1 in blocks_mod.row_blocks(tileprod[r0:r1], budget)]
        if blocks:
            # warm-up, untimed: the largest block once, so that the memory
            # pool holds a block's arrays before the timed pass (otherwise
            # the first pass's timings include growing the pool by tens of GB)
            wb0, wb1 = max(blocks, key=lambda b: int(tileprod[b[0]:b[1]].sum()))
            TA = tsg.csr_host_to_tiled(ctx, blocks_mod.block_rows(A, wb0, wb1), tsg.TSG_TILED_PACKED_COL)
            C, _ = tsg.spgemm(ctx, TA, TB)
            C.free()
            TA.free()
        ctx.set_timing(True)
        steps_ms, nnz, tiles, comp = 0.0, 0, 0, 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for b0, b1 in blocks:
            TA = tsg.csr_host_to_tiled(ctx, blocks_mod.block_rows(A, b0, b1), tsg.TSG_TILED_PACKED_COL)
            C, info = tsg.spgemm(ctx, TA, TB)
            steps_ms += info["ms_total"]
            nnz += info["nnz_C"]
            tiles += info["numtile_C"]
            comp += compulsory_bytes(TA, TB, info["numtile_C"], info["nnz_C"])
            C.free()
            TA.free()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        ctx.set_timing(False)
        TB.free()
        rows = min(r1 * 16, m) - min(r0 * 16, m)
        mine = {"tile_rows": [int(r0), int(r1)], "products": int(tileprod[r0:r1].sum()), "blocks": len(blocks),
                "ms_steps_1_3": round(steps_ms, 1)}
        if world > 1:
            ms = max_over_ranks(steps_ms, dist, device)
            wall = max_over_ranks(wall, dist, device)
            comp = sum_over_ranks(float(comp), dist, device)
            _, _, nnz_total, per = shard.global_offsets(rows, nnz, dist, device)
        else:
            ms, nnz_total, per = steps_ms, nnz, [(rows, nnz)]
        prods = int(tileprod.sum())
        out[label] = {"products": prods, "nnz_C": int(nnz_total), "tiles_C_this_rank": int(tiles),
                      "blocks_this_rank": len(blocks), "ms_steps_1_3": round(ms, 1),
                      "gflops": round(2.0 * prods / (ms * 1e-3) / 1e9, 2), "wall_s": round(wall, 2),
                      "compulsory_bytes": int(comp),
                      "hbm_frac": round(comp / (ms * 1e-3) / 1e9 / (peak * world), 4)}
        if world > 1:
            out[label]["this_rank"] = mine
            out[label]["rows_nnz_per_rank"] = per
    return out


def run_cusparse(args, mat, prods, reps=5):
    """The same product, C = A*A for the stencil, by cuSPARSE's FP64 SpGEMM
    (through torch's CUDA CSR matmul), inputs resident, CUDA-event timed: a
    library reference on the same GPU, not part of this library's path."""
    import warnings

    import torch
    m, n, rp, ci, v = mat
    dev = torch.device("cuda", torch.cuda.current_device())
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        A = torch.sparse_csr_tensor(torch.from_numpy(rp.astype(np.int64)).to(dev),
                                    torch.from_numpy(ci.astype(np.int64)).to(dev),
                                    torch.from_numpy(v).to(dev), size=(m, n))
        C = torch.sparse.mm(A, A)
        nnz = int(C._nnz())
        del C
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        best = float("inf")
        for _ in range(reps):
            torch.cuda.synchronize()
            ev[0].record()
            C = torch.sparse.mm(A, A)
            ev[1].record()
            ev[1].synchronize()
            best = min(best, ev[0].elapsed_time(ev[1]))
            del C
    return {"what": "cuSPARSE SpGEMM (torch.sparse.mm, CSR, FP64, int64 indices), same product", "ms": round(best, 3),
            "gflops": round(2.0 * prods / (best * 1e-3) / 1e9, 2), "nnz_C": nnz}


def res_name(sel, idx):
    o, a = sel.CONFIGS[idx]
    return f"{o}/{a[0]}-{a[1]}-{a[2]}"


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
    stream = torch.cuda.Stream(dev)  # one non-default stream for torch and the library
    torch.cuda.set_stream(stream)
    ctx = tsg.Context(local, stream=stream.cuda_stream)
    ctx.set_schedule(args.sched, args.seg, args.cap)
    d_rp = torch.from_numpy(rp).to(dev)
    d_ci = torch.from_numpy(ci).to(dev)
    d_v = torch.from_numpy(v).to(dev)
    A = tsg.csr_to_tiled(ctx, m, n, d_rp, d_ci, d_v, tsg.TSG_TILED_CSC_VIEW)  # serves as A and B
    prods = tsg.count_products(ctx, d_ci, d_rp)
    tiles_A = A.numtile
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
    total_ms = max_over_ranks(float(np.sum(step_ms)), dist, dev)
    ms_per_step = total_ms / args.steps
    value = replica_gflops(prods, world, ms_per_step)

    # roofline of the dominant kernel (numeric step)
    peak, peak_src = measured_peak_hbm()
    s3 = float(np.mean(s3_ms))
    alg3 = step3_algorithmic_bytes(A, A, numC, nnzC)
    achieved = alg3 / (s3 * 1e-3) / 1e9
    comp = compulsory_bytes(A, A, numC, nnzC)

    # end to end through the C ABI with host buffers: pinned inputs, results
    # written into reused pinned output buffers by one call whose copy of C
    # overlaps the numeric step (tsg_spgemm_csr_host_into)
    e2e_t, h2d, d2h = float("nan"), 0, 0
    if not args.no_e2e:
        pin = lambda x: torch.from_numpy(x).pin_memory().numpy()  # noqa: E731
        hmat = (m, n, pin(rp), pin(ci), pin(v))
        outbuf = tsg.HostResultBuffers(m, nnzC)
        tsg.spgemm_csr_host_overlap(ctx, hmat, None, outbuf)
        e2e_ms = []
        for _ in range(max(2, min(args.steps, 5))):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            Cc, _ = tsg.spgemm_csr_host_overlap(ctx, hmat, None, outbuf)
            torch.cuda.synchronize()
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
        e2e_t = float(np.mean(e2e_ms))
        h2d = rp.nbytes + ci.nbytes + v.nbytes
        d2h = Cc[2].nbytes + Cc[3].nbytes + Cc[4].nbytes
    # sections beyond the headline run on one GPU; with several ranks only the
    # row-partitioned R-MAT product runs (the stencil line above is replicas)
    sections = args.sections if world == 1 else args.sections & {"rmat20"}
    cusparse = None
    if "cusparse" in sections:
        cusparse = run_cusparse(args, mat, prods)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_reference(argparse.Namespace(warmup=0, steps=1), gen, 1, 0)
    batched = served = None
    A.free()
    if "batched" in sections:
        batched = run_batched(args, tsg, gen, ctx, max(2, min(args.steps, 5)))
    served_host = None
    if "served" in sections:
        served = run_served(args, tsg, gen, local, deliver="device")
        plain = run_served_plain(args, tsg, gen, ctx)
        served["plain_path"] = plain
        served["served_vs_plain"] = round(served["jobs_per_s"] / plain["jobs_per_s"], 3)
        served_host = run_served(args, tsg, gen, local, deliver="host", n_jobs=min(args.served_jobs, 600),
                                 half_capacity=False)
    selector = run_selector(args, tsg, gen, ctx) if "selector" in sections else None
    orderings = run_orderings(args, tsg, gen, ctx) if "orderings" in sections else None
    hyper = run_hyper(args, tsg, gen, ctx) if "hyper" in sections else None
    rmat16 = run_rmat16(args, tsg, gen, ctx) if "rmat16" in sections else None
    rmat20 = (run_rmat20(args, tsg, gen, ctx, rank=rank, world=world, dist=dist, device=dev)
              if "rmat20" in sections else None)
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "C = A*A, 27-point stencil on a 64^3 grid (n=262,144, nnz=6,859,000, FP64 "
                               "uniform(0.5,1.5)), natural order, 16x16 tiles",
                   "products": prods, "tiles_A": tiles_A, "tiles_C": numC, "nnz_C": nnzC,
                   "window": "steps 1-3 incl. C allocation (reference tilespgemm window)",
                   "schedule": f"{args.sched} seg={args.seg} cap={args.cap}",
                   "l2": "512 MiB write before every timed step, outside the timed events",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "hbm_gbs": round(comp / (ms_per_step * 1e-3) / 1e9, 2),
        "hbm_frac": round(comp / (ms_per_step * 1e-3) / 1e9 / peak, 4),
        "compulsory_bytes": comp,
        "step_ms": {k: round(float(np.mean([i[k] for i in infos])), 4) for k in ("ms_step1", "ms_step2", "ms_step3")},
        "roofline": {"bound": "hbm", "kernel": infos[-1]["step3_name"] + " (numeric step)", "achieved": round(achieved, 2),
                     "peak": peak, "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "algorithmic_bytes": alg3, "traffic": profiled_traffic("stencil27_64", args.sched)},
        "e2e": {"value": round(2.0 * prods / (e2e_t * 1e-3) / 1e9, 3), "unit": "GFLOP/s", "ms": round(e2e_t, 3),
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "path": "tsg_spgemm_csr_host_into (host CSR in -> host CSR out into the caller's pinned buffers; "
                        "the copy of C overlaps the numeric step)"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if cpu:
        out["cpu_baseline"] = cpu
    if batched:
        out["batched"] = batched
    if served:
        out["served"] = served
    if served_host:
        out["served_host_delivery"] = served_host
    if selector:
        out["selector"] = selector
    if orderings:
        out["orderings"] = orderings
    if hyper:
        out["hypersparse"] = hyper
    if rmat16:
        out["rmat16"] = rmat16
    if rmat20:
        out["rmat20_sharded" if world > 1 else "rmat20"] = rmat20
        # the second benchmark configuration beside the headline
        out["config2"] = {"workload": "R-MAT scale 20, edge factor 16: C = A*A and C = A*A^T in row blocks" +
                                      (f", row-partitioned over {world} ranks" if world > 1 else ""),
                          "gflops": {k: rmat20[k]["gflops"] for k in ("A*A", "A*A^T")},
                          "hbm_frac": {k: rmat20[k]["hbm_frac"] for k in ("A*A", "A*A^T")},
                          "scaling": "strong" if world > 1 else None}
    if cusparse:
        out["library_reference"] = cusparse
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
    ap.add_argument("--sched", default="spa", choices=["rows", "tiles", "elems", "spa"])
    ap.add_argument("--sections", default="plain,cusparse,batched,served,orderings,hyper,rmat20,selector",
                    help="comma list: plain (always), cusparse, batched, served, orderings, hyper, rmat16, rmat20, "
                         "selector")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--selector-samples", type=int, default=5000)
    ap.add_argument("--served-jobs", type=int, default=2000)
    ap.add_argument("--served-rate", type=float, default=2000.0)
    ap.add_argument("--served-schedule", default="auto",
                    help='"auto" (tuned per density class) or schedule,seg,cap[,dense], e.g. spa,8,512')
    ap.add_argument("--seg", type=int, default=16)
    ap.add_argument("--cap", type=int, default=1024)
    args = ap.parse_args()
    args.sections = set(args.sections.split(","))
    if args.served_schedule != "auto":
        f = args.served_schedule.split(",")
        args.served_schedule = (f[0],) + tuple(int(x) for x in f[1:])
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
