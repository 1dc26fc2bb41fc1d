"""Row blocks of A for products larger than one device, and their partition
over ranks.

Rows of C depend only on the matching rows of A and on all of B, so C = A*B
can be computed one block of A's tile rows at a time against a resident B
(its C freed or kept per block), and a block list can be split over ranks
with B replicated in each rank's memory and no exchange inside the product.
Work is measured in scalar products (sum over A's entries (i, k) of nnz(B
row k), the reference's nnzCub of src/main.cu:392-397) per tile row of A --
the quantity the step-1 count bounds and the numeric step's time follows.
"""
from __future__ import annotations

import numpy as np

TILE = 16


def tile_row_products(matA, matB) -> np.ndarray:
    """Scalar products of every 16-row tile row of A (int64)."""
    m, _, rp, ci, _ = matA
    rpB = np.asarray(matB[2], dtype=np.int64)
    blen = np.diff(rpB)
    rp = np.asarray(rp, dtype=np.int64)
    rowprod = np.zeros(m, np.int64)
    nz = np.diff(rp) > 0
    if nz.any():
        rowprod[nz] = np.add.reduceat(blen[np.asarray(ci)], rp[:-1][nz])
    tilem = (m + TILE - 1) // TILE
    if m == 0:
        return np.zeros(0, np.int64)
    return np.add.reduceat(rowprod, np.arange(0, m, TILE))[:tilem]


def row_blocks(tile_prods: np.ndarray, budget: float) -> list[tuple[int, int]]:
    """Consecutive tile-row blocks [t0, t1) of at most `budget` products each
    (a tile row above the budget is a block alone)."""
    bounds, acc = [0], 0
    for t, pt in enumerate(tile_prods):
        if acc > 0 and acc + pt > budget:
            bounds.append(t)
            acc = 0
        acc += int(pt)
    bounds.append(len(tile_prods))
    return [(a, b) for a, b in zip(bounds[:-1], bounds[1:]) if b > a]


def partition(tile_prods: np.ndarray, parts: int) -> list[tuple[int, int]]:
    """`parts` consecutive tile-row ranges [t0, t1) covering every tile row
    once, cut where the running product count crosses k/parts of the total
    (each range within one tile row's work of an equal share)."""
    tilem = len(tile_prods)
    if parts <= 1 or tilem == 0:
        return [(0, tilem)] + [(tilem, tilem)] * max(parts - 1, 0)
    csum = np.concatenate([[0], np.cumsum(tile_prods, dtype=np.int64)])
    total = csum[-1]
    cuts = [0]
    for k in range(1, parts):
        want = total * k / parts
        t = int(np.searchsorted(csum, want, side="left"))
        # nearer of the two tile-row boundaries around the share
        if t > 0 and abs(csum[t - 1] - want) <= abs(csum[min(t, tilem)] - want):
            t -= 1
        cuts.append(min(max(t, cuts[-1]), tilem))
    cuts.append(tilem)
    return list(zip(cuts[:-1], cuts[1:]))


def block_rows(matA, t0: int, t1: int):
    """The CSR block of A's rows [16 t0, 16 t1) (rows renumbered from 0)."""
    m, n, rp, ci, v = matA
    r0, r1 = min(t0 * TILE, m), min(t1 * TILE, m)
    return (r1 - r0, n, (np.asarray(rp[r0:r1 + 1]) - rp[r0]).astype(np.int32), np.asarray(ci[rp[r0]:rp[r1]]),
            np.asarray(v[rp[r0]:rp[r1]]))
