"""Autotuner for the batched and one-product tiled SpGEMM.

For a batch (or one product) it times every candidate configuration -- work
schedule of steps 2-3 (sparse accumulator / tile / element / row-segment),
the row schedule's segment length (C tiles per work item) and its FP64
accumulator capacity, and the sparse accumulator's dense threshold (C values
per tile from which a product's numeric step takes the tile kernel), which
together set the block schedule and the sparse/dense accumulator split --
and keeps the fastest.  A candidate is (schedule, seg_tiles, acc_cap,
dense); dense 0 is the default threshold and is ignored by the other
schedules.
Winners are cached by a key of batch features (product count, total scalar
products, mean nonzeros per C-tile bound), in memory and optionally in a
JSON file, so a similar batch reuses the choice without timing.

The tile size itself is fixed at 16x16: the format's 16-bit row masks and
4-bit in-tile columns, and bit-exact parity with the reference, are defined
for 16 only.  All candidates return bit-identical results, so the choice
affects time only.
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

from . import Batch, Context, product_bounds, spgemm

CANDIDATES = [("spa", 8, 512, 0), ("spa", 8, 512, 32), ("spa", 8, 512, 128), ("spa", 8, 512, 257),
              ("elems", 8, 512, 0), ("tiles", 8, 512, 0), ("rows", 16, 1024, 0), ("rows", 8, 256, 0),
              ("rows", 32, 2048, 0)]


def normalize(cand) -> tuple:
    """(schedule, seg_tiles, acc_cap, dense) from a 3- or 4-entry candidate."""
    c = tuple(cand)
    return c + (0,) if len(c) == 3 else c


def make_batch(ctx: Context, pairs, cand, graph: bool = True) -> Batch:
    s, w, c, d = normalize(cand)
    return Batch(ctx, pairs, s, w, c, graph=graph, dense=d)


def batch_key(ctx: Context, pairs) -> str:
    prods, tiles = 0, 0
    for A, B in pairs:
        p, t = product_bounds(ctx, A, B)
        prods += p
        tiles += t
    dens = prods / max(tiles, 1)
    return f"n{int(math.log2(len(pairs) + 1))}-p{int(math.log2(prods + 1))}-d{int(math.log2(dens + 1))}"


class Autotuner:
    def __init__(self, cache_path: str | None = None, candidates=None):
        self.candidates = [normalize(c) for c in (candidates or CANDIDATES)]
        self.path = Path(cache_path) if cache_path else None
        self.cache = {}
        if self.path and self.path.exists():
            self.cache = {k: normalize(v) for k, v in json.loads(self.path.read_text()).items()}
        self.last_timings = {}

    def _save(self):
        if self.path:
            self.path.write_text(json.dumps(self.cache, indent=1))

    def tune_batch(self, ctx: Context, pairs, reps: int = 2, use_cache: bool = True):
        """Best (schedule, seg_tiles, acc_cap, dense) for this batch; timings
        in self.last_timings (ms per run)."""
        import torch
        key = "batch-" + batch_key(ctx, pairs)
        if use_cache and key in self.cache:
            return self.cache[key]
        timings = {}
        for cand in self.candidates:
            b = make_batch(ctx, pairs, cand, graph=True)
            b.run()
            b.sync()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            stream = torch.cuda.current_stream()
            best = float("inf")
            for _ in range(reps):
                ctx.synchronize()
                ev[0].record(stream)
                b.run()
                ctx.synchronize()
                ev[1].record(stream)
                ev[1].synchronize()
                best = min(best, ev[0].elapsed_time(ev[1]))
            b.sync()
            b.close()
            timings[cand] = best
        choice = min(timings, key=timings.get)
        self.last_timings = timings
        self.cache[key] = choice
        self._save()
        return choice

    def tune_single(self, ctx: Context, A, B, reps: int = 2, use_cache: bool = True):
        """Best schedule for one product on the one-product path."""
        key = "single-" + batch_key(ctx, [(A, B)])
        if use_cache and key in self.cache:
            return self.cache[key]
        ctx.set_timing(True)
        timings = {}
        for cand in self.candidates:
            ctx.set_schedule(*cand)
            best = float("inf")
            for _ in range(reps + 1):
                C, info = spgemm(ctx, A, B)
                best = min(best, info["ms_total"])
                C.free()
            timings[cand] = best
        ctx.set_timing(False)
        choice = min(timings, key=timings.get)
        ctx.set_schedule(*choice)
        self.last_timings = timings
        self.cache[key] = choice
        self._save()
        return choice


def label(cand) -> str:
    s, w, c, d = normalize(cand)
    return f"{s}-{w}-{c}" + (f"-d{d or 64}" if s == "spa" else "")


def summarize(timings: dict) -> dict:
    return {label(k): round(t, 4) for k, t in timings.items()}


__all__ = ["Autotuner", "CANDIDATES", "batch_key", "label", "make_batch", "normalize", "summarize", "np"]
