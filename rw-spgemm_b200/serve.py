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
import math
import threading
import time
from concurrent.futures import Future

import numpy as np

from . import TSG_TILED_CSC_VIEW, Batch, Context, check, csr_host_to_tiled, lib, product_bounds


class Job:
    __slots__ = ("jid", "kind", "a_key", "b_key", "t_submit", "t_done", "future", "pred_bytes", "pred_prods",
                 "pred_tiles", "result_nnz")

    def __init__(self, jid, kind, a_key, b_key):
        self.jid, self.kind, self.a_key, self.b_key = jid, kind, a_key, b_key
        self.t_submit = time.perf_counter()
        self.t_done = None
        self.future = Future()
        self.pred_bytes = 0
        self.pred_prods = 0
        self.pred_tiles = 0
        self.result_nnz = 0


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
        self.ctx = Context(device, own_stream=True)
        self.staging = None  # page-locked result staging, grown on demand
        self.batch = None
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
    schedule  (schedule, seg_tiles, acc_cap[, dense]) of the batched kernel,
              or "auto": the autotuner (`tuner`, a fresh one if None)
              times its candidates on the first batch of each density class
              and the class keeps that choice
    deliver   "host": a job's result is (m, n, rowptr, colidx, val) as numpy
              arrays; "device": the same as torch tensors on the GPU (for a
              consumer that stays on the device; nothing crosses the bus)
    """

    def __init__(self, device=0, mem_cap=40 << 30, slots=2, max_batch=64, schedule=("spa", 8, 512),
                 batch_products=2e8, deliver="host", tuner=None):
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

    # -- registration / submission -------------------------------------------
    def register(self, key, mat):
        self.matrices[key] = mat

    def submit(self, kind, a_key, b_key=None) -> Future:
        if kind not in ("AB", "AAT"):
            raise ValueError(kind)
        if kind == "AAT":
            tkey = (a_key, "T")
            if tkey not in self.matrices:
                self.matrices[tkey] = _transpose(self.matrices[a_key])
            b_key = tkey
        with self.lock:
            job = Job(self.next_id, kind, a_key, b_key)
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
        for t in self.cache.tiles.values():
            t.free()
        self.cache.tiles.clear()
        for s in self.slots:
            s.ctx.close()
        self.stage_ctx.close()

    # -- dispatcher ----------------------------------------------------------------
    def _in_use(self):
        return self.cache.bytes + sum(s.arena for s in self.slots if s.batch is not None)

    def _predict(self, A, B):
        """(device bytes of the result arena, scalar products, C-tile bound)
        from the step-1 bounds; the arena's per-array 256-byte alignment
        and per-tile-row flags included."""
        prods, pairs = product_bounds(self.cache.ctx, A, B)
        tiles = min(pairs, A.s.tilem * B.s.tilen)
        vals = min(prods, 256 * tiles)
        return (tiles * (4 * 3 + 4 + 32 + 16) + vals * 9 + (A.s.tilem + 1) * 4 + A.s.tilem * 4 + 8 * 256,
                prods, tiles)

    def _schedule_for(self, slot, pairs, jobs):
        """The batch's (schedule, seg_tiles, acc_cap, dense)."""
        if self.schedule != "auto":
            s = tuple(self.schedule)
            return s + (0,) if len(s) == 3 else s
        prods = sum(j.pred_prods for j in jobs)
        tiles = max(1, sum(j.pred_tiles for j in jobs))
        key = int(math.log2(prods / tiles + 1))
        if key not in self.tuned:
            self.tuned[key] = self.tuner.tune_batch(slot.ctx, pairs, reps=1, use_cache=False)
        return self.tuned[key]

    def _form_batch(self, slot):
        jobs, pairs, pred, work = [], [], 0, 0
        # operands of batches still running must stay resident
        pinned = {k for s in self.slots if s.batch is not None for j in s.jobs for k in (j.a_key, j.b_key)}
        while self.queue and len(jobs) < self.max_batch:
            job = self.queue[0]
            A = self.cache.get(job.a_key, self.matrices[job.a_key])
            B = self.cache.get(job.b_key, self.matrices[job.b_key])
            job.pred_bytes, job.pred_prods, job.pred_tiles = self._predict(A, B)
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
        if not jobs:
            return False
        sch, seg, cap, dense = self._schedule_for(slot, pairs, jobs)
        slot.batch = Batch(slot.ctx, pairs, sch, seg, cap, graph=False, dense=dense)
        slot.arena = slot.batch.info()["arena_bytes"]
        slot.jobs = jobs
        slot.t_launch = time.perf_counter()
        slot.batch.run()
        self.batches += 1
        return True

    def _finish(self, slot):
        """Converts every product of the finished batch to CSR on the device
        (all conversions queued on the slot's stream, one synchronisation).
        deliver="device": each job gets its device tensors.  deliver="host":
        the batch's results go through the slot's reusable page-locked
        staging buffer (one copy; pinning fresh memory per batch costs more)
        into numpy arrays of each job."""
        import torch
        slot.batch.sync()
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
        dbuf = torch.empty(max(total, 8), dtype=torch.uint8, device=dev)
        base = dbuf.data_ptr()
        for job, C, m, n, nnz, v_off, rp_off, ci_off in layout:
            check(lib().tsg_tiled_to_csr(slot.ctx.handle, ctypes.byref(C.s), ctypes.c_void_p(base + rp_off),
                                         ctypes.c_void_p(base + ci_off), ctypes.c_void_p(base + v_off)))
        slot.ctx.synchronize()
        if self.deliver == "device":
            for job, C, m, n, nnz, v_off, rp_off, ci_off in layout:
                res = (m, n, dbuf[rp_off:rp_off + 4 * (m + 1)].view(torch.int32),
                       dbuf[ci_off:ci_off + 4 * nnz].view(torch.int32), dbuf[v_off:v_off + 8 * nnz].view(torch.float64))
                self._complete(job, nnz, res)
        else:
            if slot.staging is None or slot.staging.numel() < total:
                slot.staging = torch.empty(max(total, 1 << 20), dtype=torch.uint8, pin_memory=True)
            slot.staging[:max(total, 8)].copy_(dbuf)
            raw = slot.staging.numpy()
            for job, C, m, n, nnz, v_off, rp_off, ci_off in layout:
                res = (m, n, raw[rp_off:rp_off + 4 * (m + 1)].view(np.int32).copy(),
                       raw[ci_off:ci_off + 4 * nnz].view(np.int32).copy(), raw[v_off:v_off + 8 * nnz].view(np.float64).copy())
                self._complete(job, nnz, res)
        self._release(slot)

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
                    self._finish(slot)
                    progressed = True
            for slot in self.slots:
                if slot.batch is None and self.queue:
                    progressed |= self._form_batch(slot)
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
        }
