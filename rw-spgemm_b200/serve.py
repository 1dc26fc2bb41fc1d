"""Serving layer: a continuous-batching request loop over the batched engine.

Jobs (C = A*B or C = A*A^T over registered matrices) arrive at any time.  A
dispatcher thread
  * keeps every operand resident on the device as tiles (one tiled copy per
    matrix serves both the A and B roles; A^T is registered on first use) in
    an LRU cache,
  * admits queued jobs in arrival order while the device memory in use --
    resident operands + result arenas of batches in flight + the new job's
    predicted bytes -- stays under the cap; the prediction comes from the
    job's step-1/step-2 bounds on the device (matched tile pairs, scalar
    products),
  * packs admitted jobs into a batch (tsg_batch: one persistent,
    graph-captured launch) on a free stream slot while earlier batches are
    still running on the other slots, so their work overlaps on the GPU,
    with the batch schedule fixed or (schedule="auto") chosen by the
    autotuner once per density class of batch (scalar products per C-tile
    bound, in powers of two) and reused for every later batch of the class,
  * when a batch finishes, copies each result to host CSR and completes the
    job's future with its latency (submit -> result on the host).
Results are bit-identical whether a job runs alone or inside any mix: each
output entry is accumulated in a fixed order independent of batching.
"""
from __future__ import annotations

import collections
import ctypes
import itertools
import math
import os
import threading
import time
from concurrent.futures import Future

import numpy as np

from . import (TSG_TILED_CSC_VIEW, Batch, Context, check, csr_host_to_tiled, lib, product_bounds,
               product_bounds_many)


class Job:
    __slots__ = ("jid", "kind", "a_key", "b_key", "cls", "t_submit", "t_done", "future", "pred_bytes",
                 "pred_prods", "pred_tiles", "result_nnz")

    def __init__(self, jid, kind, a_key, b_key, cls=0):
        self.jid, self.kind, self.a_key, self.b_key, self.cls = jid, kind, a_key, b_key, cls
        self.t_submit = time.perf_counter()
        self.t_done = None
        self.future = Future()
        self.pred_bytes = 0
        self.pred_prods = -1  # not predicted yet
        self.pred_tiles = 0
        self.result_nnz = 0


def skew_class(mat):
    """floor(log2(longest row / mean row)) of a host CSR (0 when empty):
    products whose A rows are this uneven take about as long to finish
    their heaviest rows, so batches of one class overlap their tails."""
    m, n, rp, ci, v = mat
    d = np.diff(np.asarray(rp, dtype=np.int64))
    if m == 0 or d.sum() == 0:
        return 0
    return int(math.log2(max(1.0, float(d.max()) / float(d.mean()))))


def _transpose(mat):
    m, n, rp, ci, v = mat
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(rp))
    order = np.lexsort((rows, ci))
    rp_t = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rp_t, ci.astype(np.int64) + 1, 1)
    return n, m, np.cumsum(rp_t).astype(np.int32), rows[order].astype(np.int32), np.asarray(v)[order]


class OperandCache:
    """Device-resident tiled operands (row tiles + column view), LRU."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.tiles = collections.OrderedDict()
        self.bytes = 0
        self.hits = 0
        self.misses = 0

    @staticmethod
    def tiled_bytes(t):
        """Device bytes of a resident operand, as the library allocated them:
        tiles, column view, column masks and the row view of the B role."""
        return t.device_bytes

    def get(self, key, host_mat):
        if key in self.tiles:
            self.tiles.move_to_end(key)
            self.hits += 1
            return self.tiles[key]
        self.misses += 1
        t = csr_host_to_tiled(self.ctx, host_mat, TSG_TILED_CSC_VIEW)
        self.tiles[key] = t
        self.bytes += self.tiled_bytes(t)
        return t

    def size_of(self, key):
        """Device bytes of a resident operand."""
        return self.tiled_bytes(self.tiles[key])

    def drop(self, keys):
        for key in keys:
            t = self.tiles.pop(key, None)
            if t is not None:
                self.bytes -= self.tiled_bytes(t)
                t.free()

    def evict_until(self, limit, pinned_keys):
        for key in list(self.tiles.keys()):
            if self.bytes <= limit:
                break
            if key in pinned_keys:
                continue
            t = self.tiles.pop(key)
            self.bytes -= self.tiled_bytes(t)
            t.free()


class _Slot:
    """One in-flight batch position with its own stream."""

    def __init__(self, device):
        import torch
        # a torch stream (non-blocking), so that torch copies of the results
        # queue behind the library's work on it
        self.stream = torch.cuda.Stream(device)
        self.ctx = Context(device, stream=self.stream.cuda_stream)
        self.staging = None  # page-locked result staging, grown on demand
        self.batch = None
        self.pending = None  # conversions queued, results not yet handed over
        self.jobs = []
        self.arena = 0
        self.t_launch = 0.0

    def idle_stream(self) -> bool:
        return lib().tsg_context_query(self.ctx.handle) == 0


class SpGEMMServer:
    """Continuous-batching SpGEMM server on one GPU.

    mem_cap   bytes of device memory the server may hold (operands + arenas)
    slots     batches that may be in flight at once (one stream each)
    max_batch jobs per batch
    batch_products  scalar-product budget of a batch (the jobs' step-1
              bounds): a batch closes once it holds this much work, so a few
              large jobs do not hold many small ones back (a single job
              above it still runs, alone)
    A batch takes the first queued job and the later jobs of the same skew
    class (skew_class of the A operand) among the next 4 * max_batch queued,
    in arrival order; jobs of other classes keep their places.  Products of
    one class finish their heaviest rows at about the same time, so a batch
    does not wait on one skewed product's tail while the GPU idles.
    schedule  (schedule, seg_tiles, acc_cap[, dense]) of the batched kernel,
              or "auto": the autotuner (`tuner`, a fresh one if None)
              times its candidates on the first batch of each density class
              and the class keeps that choice
    deliver   "host": a job's result is (m, n, rowptr, colidx, val) as numpy
              arrays; "device": the same as torch tensors on the GPU (for a
              consumer that stays on the device; nothing crosses the bus)
    """

    def __init__(self, device=0, mem_cap=40 << 30, slots=2, max_batch=64, schedule=("spa", 8, 512),
                 batch_products=5e8, deliver="host", tuner=None):
        if deliver not in ("host", "device"):
            raise ValueError(deliver)
        self.deliver = deliver
        self.device = device
        self.mem_cap = int(mem_cap)
        self.max_batch = max_batch
        self.batch_products = float(batch_products)
        self.schedule = schedule
        self.tuner = tuner
        self.tuned = {}  # density class -> chosen schedule ("auto")
        if schedule == "auto" and self.tuner is None:
            from .autotune import Autotuner
            self.tuner = Autotuner()
        self.matrices = {}
        self.slots = [_Slot(device) for _ in range(slots)]
        self.stage_ctx = Context(device, own_stream=True)  # operand staging and bounds
        self.cache = OperandCache(self.stage_ctx)
        self.queue = collections.deque()
        self.lock = threading.Condition()
        self.running = False
        self.thread = None
        self.next_id = 0
        self.done = []
        self.batches = 0
        self.rejected = 0
        self.preds = {}  # (a_key, b_key) -> (arena bytes, scalar products, C tiles)
        self.classes = {}  # operand key -> skew_class of the matrix
        self.lookahead = 4 * max_batch  # queued jobs a batch may look through for its class
        # dispatcher time by activity ("form" includes tune, predict, create
        # and run); "gpu": the batches' kernel time, from their device timer
        # stamps
        self.host_s = {"form": 0.0, "tune": 0.0, "predict": 0.0, "create": 0.0, "run": 0.0, "finish": 0.0,
                       "deliver": 0.0, "gpu": 0.0}

    # -- registration / submission -------------------------------------------
    def register(self, key, mat):
        """Registers operand `key`.  Replacing one drops what was derived from
        the old matrix (its transpose, bounds and resident tiles); an operand
        of a queued or running job cannot be replaced."""
        if key in self.matrices and self.matrices[key] is not mat:
            keys = {key, (key, "T")}
            busy = [j for j in self.queue] + [j for sl in self.slots for j in sl.jobs]
            if any(j.a_key in keys or j.b_key in keys for j in busy):
                raise RuntimeError(f"operand {key!r} is in use by a queued or running job")
            self.matrices.pop((key, "T"), None)
            self.preds = {k: v for k, v in self.preds.items() if not (set(k) & keys)}
            self.cache.drop(keys)
        self.matrices[key] = mat
        self.classes[key] = skew_class(mat)

    def submit(self, kind, a_key, b_key=None) -> Future:
        if kind not in ("AB", "AAT"):
            raise ValueError(kind)
        if kind == "AAT":
            tkey = (a_key, "T")
            if tkey not in self.matrices:
                self.matrices[tkey] = _transpose(self.matrices[a_key])
            b_key = tkey
        with self.lock:
            job = Job(self.next_id, kind, a_key, b_key, self.classes.get(a_key, 0))
            self.next_id += 1
            self.queue.append(job)
            self.lock.notify()
        return job.future

    # -- lifecycle ---------------------------------------------------------------
    def start(self):
        self.running = True
        self.thread = threading.Thread(target=self._loop, name="spgemm-dispatch", daemon=True)
        self.thread.start()
        return self

    def stop(self, drain=True):
        if drain:
            while True:
                with self.lock:
                    idle = not self.queue and all(s.batch is None for s in self.slots)
                if idle:
                    break
                time.sleep(0.0005)
        self.running = False
        with self.lock:
            self.lock.notify()
        if self.thread:
            self.thread.join()
        for s in self.slots:
            if s.batch is not None:
                s.batch.close()
            s.ctx.synchronize()

    def close(self):
        self.stop()
        if getattr(self, "_pool", None) is not None:
            self._pool.shutdown()
            self._pool = None
        for t in self.cache.tiles.values():
            t.free()
        self.cache.tiles.clear()
        for s in self.slots:
            s.ctx.close()
        self.stage_ctx.close()

    # -- dispatcher ----------------------------------------------------------------
    def _in_use(self):
        return self.cache.bytes + sum(s.arena for s in self.slots if s.batch is not None)

    @staticmethod
    def _arena_of(A, prods, ctiles):
        """Device bytes of a product's share of the batch arena, laid out as
        tsg_batch_create does (row offsets and flags per A tile row, C's tile
        arrays for ctiles tiles, min(products, 256 ctiles) values; every
        array 256-byte aligned)."""
        def al(x):
            return (x + 255) & ~255
        tm = A.s.tilem
        vals = min(prods, 256 * ctiles)
        return (al((tm + 1) * 4) + al(tm * 4) + 2 * al(ctiles * 4) + al((ctiles + 1) * 4) + al(ctiles * 32) +
                al(ctiles * 16) + al(vals) + al(vals * 8))

    def _predict_many(self, ops):
        """(arena bytes, scalar products, C tiles) of each (A, B), with one
        synchronisation (step 1's exact C-tile count)."""
        return [(self._arena_of(A, prods, ctiles), prods, ctiles)
                for (A, B), (prods, _, ctiles) in zip(ops, product_bounds_many(self.cache.ctx, ops, c_tiles=True))]

    def _predict(self, A, B):
        return self._predict_many([(A, B)])[0]

    def _predict_jobs(self, jobs, ops):
        """Fills the jobs' predictions: from the cache of earlier jobs on the
        same operand pair, the others with one call."""
        need = {}
        for j, op in zip(jobs, ops):
            if (j.a_key, j.b_key) not in self.preds:
                need.setdefault((j.a_key, j.b_key), op)
        if need:
            keys = list(need)
            preds = ([self._predict(*need[keys[0]])] if len(keys) == 1 else
                     self._predict_many([need[k] for k in keys]))
            self.preds.update(zip(keys, preds))
        for j in jobs:
            j.pred_bytes, j.pred_prods, j.pred_tiles = self.preds[(j.a_key, j.b_key)]

    def _predict_queue(self):
        """Predicts the queued jobs of the first job's class within the
        lookahead (as many as a batch holds) whose operands are resident,
        with at most one synchronisation."""
        cls = self.queue[0].cls if self.queue else 0
        todo = [j for j in itertools.islice(self.queue, self.lookahead) if j.cls == cls and j.pred_prods < 0 and
                j.a_key in self.cache.tiles and j.b_key in self.cache.tiles][:self.max_batch]
        if todo:
            self._predict_jobs(todo, [(self.cache.tiles[j.a_key], self.cache.tiles[j.b_key]) for j in todo])

    def _schedule_for(self, slot, pairs, jobs):
        """The batch's (schedule, seg_tiles, acc_cap, dense)."""
        if self.schedule != "auto":
            s = tuple(self.schedule)
            return s + (0,) if len(s) == 3 else s
        prods = sum(j.pred_prods for j in jobs)
        tiles = max(1, sum(j.pred_tiles for j in jobs))
        key = int(math.log2(prods / tiles + 1))
        if key not in self.tuned:
            t0 = time.perf_counter()
            self.tuned[key] = self.tuner.tune_batch(slot.ctx, pairs, reps=1, use_cache=False)
            self.host_s["tune"] += time.perf_counter() - t0
        return self.tuned[key]

    def _form_batch(self, slot):
        jobs, pairs, pred, work = [], [], 0, 0
        # operands of batches still running must stay resident
        pinned = {k for s in self.slots if s.batch is not None for j in s.jobs for k in (j.a_key, j.b_key)}
        t0 = time.perf_counter()
        self._predict_queue()
        self.host_s["predict"] += time.perf_counter() - t0
        # the batch takes the queue's first job and then, in arrival order,
        # the later jobs of its class within the lookahead (the others keep
        # their places)
        cls = self.queue[0].cls if self.queue else 0
        passed = []
        while self.queue and len(jobs) < self.max_batch and len(passed) < self.lookahead:
            job = self.queue[0]
            if job.cls != cls:
                passed.append(self.queue.popleft())
                continue
            A = self.cache.get(job.a_key, self.matrices[job.a_key])
            B = self.cache.get(job.b_key, self.matrices[job.b_key])
            if job.pred_prods < 0:
                self._predict_jobs([job], [(A, B)])
            if jobs and work + job.pred_prods > self.batch_products:
                break  # the batch holds its share of work; this job opens the next
            # its operands stay resident while it runs: a job needing more
            # than the cap with them could never be admitted
            need = job.pred_bytes + self.cache.size_of(job.a_key) + (
                self.cache.size_of(job.b_key) if job.b_key != job.a_key else 0)
            if need > self.mem_cap:
                self.queue.popleft()
                self.rejected += 1
                job.future.set_exception(MemoryError(f"job {job.jid} needs {need} bytes with its operands, "
                                                     f"cap {self.mem_cap}"))
                continue
            if self._in_use() + pred + job.pred_bytes > self.mem_cap:
                # evict operands of nobody running or admitted (this job's own kept)
                self.cache.evict_until(self.mem_cap - pred - job.pred_bytes -
                                       sum(s.arena for s in self.slots if s.batch is not None),
                                       pinned | {job.a_key, job.b_key})
                if self._in_use() + pred + job.pred_bytes > self.mem_cap:
                    break  # wait for memory to free up (arrival order kept)
            pinned.update((job.a_key, job.b_key))
            self.queue.popleft()
            jobs.append(job)
            pairs.append((A, B))
            pred += job.pred_bytes
            work += job.pred_prods
        self.queue.extendleft(reversed(passed))
        if not jobs:
            return False
        sch, seg, cap, dense = self._schedule_for(slot, pairs, jobs)
        # planned from the predictions (exact C-tile counts): no device wait
        # while the other slot's batch holds the GPU
        t0 = time.perf_counter()
        slot.batch = Batch(slot.ctx, pairs, sch, seg, cap, graph=False, dense=dense,
                           bounds=[(j.pred_prods, j.pred_tiles) for j in jobs])
        slot.arena = slot.batch.info()["arena_bytes"]
        slot.jobs = jobs
        t1 = slot.t_launch = time.perf_counter()
        slot.batch.run()
        self.host_s["create"] += t1 - t0
        self.host_s["run"] += time.perf_counter() - t1
        self.batches += 1
        return True

    def _finish(self, slot):
        """Stage 1, once the batch's stream is idle: reads the products'
        sizes and queues every conversion to CSR on the slot's stream, into
        one device buffer (and, deliver="host", its copy into the slot's
        reusable page-locked staging buffer), without waiting: the work runs
        when the GPU is free and _deliver hands the results over."""
        import torch
        slot.batch.sync()
        self.host_s["gpu"] += sum(slot.batch.phase_ms().values()) * 1e-3
        dev = torch.device("cuda", self.device)
        layout, total = [], 0
        for p, job in enumerate(slot.jobs):
            C = slot.batch.product(p)
            m, nnz = C.s.m, C.s.nnz
            v_off = total
            rp_off = v_off + 8 * nnz
            ci_off = rp_off + 4 * (m + 1)
            total = (ci_off + 4 * nnz + 7) & ~7
            layout.append((job, C, m, C.s.n, nnz, v_off, rp_off, ci_off))
        with torch.cuda.stream(slot.stream):
            dbuf = torch.empty(max(total, 8), dtype=torch.uint8, device=dev)
        base = dbuf.data_ptr()
        for job, C, m, n, nnz, v_off, rp_off, ci_off in layout:
            check(lib().tsg_tiled_to_csr(slot.ctx.handle, ctypes.byref(C.s), ctypes.c_void_p(base + rp_off),
                                         ctypes.c_void_p(base + ci_off), ctypes.c_void_p(base + v_off)))
        if self.deliver == "host":
            if slot.staging is None or slot.staging.numel() < total:
                slot.staging = torch.empty(max(total, 1 << 20), dtype=torch.uint8, pin_memory=True)
            with torch.cuda.stream(slot.stream):
                slot.staging[:max(total, 8)].copy_(dbuf, non_blocking=True)
        slot.pending = (layout, dbuf)

    def _deliver(self, slot):
        """Stage 2, once the conversions (and copies) have run: hands each
        job its result and releases the batch."""
        import torch
        layout, dbuf = slot.pending
        if self.deliver == "device":
            for job, C, m, n, nnz, v_off, rp_off, ci_off in layout:
                res = (m, n, dbuf[rp_off:rp_off + 4 * (m + 1)].view(torch.int32),
                       dbuf[ci_off:ci_off + 4 * nnz].view(torch.int32), dbuf[v_off:v_off + 8 * nnz].view(torch.float64))
                self._complete(job, nnz, res)
        else:
            # the results leave the reusable staging buffer for arrays of
            # their own; the copies (and the first touch of the new pages)
            # run on the host pool's threads, in pieces of at most 16 MB
            raw = slot.staging.numpy()
            outs, pieces = [], []
            for job, C, m, n, nnz, v_off, rp_off, ci_off in layout:
                arrs = []
                for off, count, dt in ((rp_off, m + 1, np.int32), (ci_off, nnz, np.int32), (v_off, nnz, np.float64)):
                    src = raw[off:off + count * np.dtype(dt).itemsize].view(dt)
                    dst = np.empty(count, dt)
                    step = max(1, (16 << 20) // np.dtype(dt).itemsize)
                    pieces += [(dst, src, q, min(count, q + step)) for q in range(0, count, step)]
                    arrs.append(dst)
                outs.append((job, nnz, (m, n, *arrs)))
            list(self._host_pool().map(lambda t: np.copyto(t[0][t[2]:t[3]], t[1][t[2]:t[3]]), pieces))
            for job, nnz, res in outs:
                self._complete(job, nnz, res)
        slot.pending = None
        self._release(slot)

    def _host_pool(self):
        if getattr(self, "_pool", None) is None:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(max_workers=max(1, min(16, (os.cpu_count() or 2) // 2)))
        return self._pool

    def _complete(self, job, nnz, res):
        job.t_done = time.perf_counter()
        job.result_nnz = nnz
        job.future.set_result(res)
        self.done.append(job)

    def _release(self, slot):
        slot.batch.close()
        slot.batch = None
        slot.jobs = []
        slot.arena = 0

    def _loop(self):
        # only this thread consumes the queue (deque appends/pops are atomic)
        while self.running:
            progressed = False
            for slot in self.slots:
                if slot.batch is not None and slot.idle_stream():
                    t0 = time.perf_counter()
                    stage = "finish" if slot.pending is None else "deliver"
                    (self._finish if slot.pending is None else self._deliver)(slot)
                    self.host_s[stage] += time.perf_counter() - t0
                    progressed = True
            for slot in self.slots:
                if slot.batch is None and self.queue:
                    t0 = time.perf_counter()
                    progressed |= self._form_batch(slot)
                    self.host_s["form"] += time.perf_counter() - t0
            if not progressed:
                with self.lock:
                    if not self.queue and all(s.batch is None for s in self.slots):
                        self.lock.wait(timeout=0.002)
                time.sleep(0.0001)

    # -- statistics ----------------------------------------------------------------
    def stats(self):
        lat = np.array([(j.t_done - j.t_submit) * 1e3 for j in self.done]) if self.done else np.zeros(0)
        t0 = min((j.t_submit for j in self.done), default=0.0)
        t1 = max((j.t_done for j in self.done), default=0.0)
        return {
            "jobs": len(self.done),
            "jobs_per_s": len(self.done) / (t1 - t0) if t1 > t0 else 0.0,
            "p50_ms": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_ms": float(np.percentile(lat, 99)) if lat.size else None,
            "batches": self.batches,
            "mean_batch": len(self.done) / self.batches if self.batches else 0.0,
            "rejected": self.rejected,
            "operand_cache": {"hits": self.cache.hits, "misses": self.cache.misses, "bytes": self.cache.bytes},
            "tuned": {f"d{k}": "-".join(str(x) for x in v) for k, v in sorted(self.tuned.items())},
            "dispatcher_s": {k: round(v, 4) for k, v in self.host_s.items()},
        }
