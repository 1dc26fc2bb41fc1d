"""Row-partitioned product over ranks (one process per GPU).

C = A*B is split by A's tile rows: rank r owns the consecutive tile-row range
partition(tile_prods, world)[r] of A, cut by predicted scalar products (the
step-1 work measure of blocks.py, the reference's nnzCub per row,
src/main.cu:392-397), and holds all of B in its own memory.  Rows of C depend
only on the matching rows of A and on B, so the product has no exchange step;
each rank computes its range block by block (blocks.row_blocks) and keeps its
piece of C.  The one collective is an all-gather of every rank's (rows, nnz)
after the product, which gives each rank the global row and nonzero offsets
of its piece, i.e. where it sits in the distributed CSR of C.

No kernel reads another GPU's memory: B is replicated by each rank from the
host, and the all-gather moves two integers per rank.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import blocks


@dataclass
class Piece:
    """One rank's share of C: tile rows [t0, t1) of A, i.e. global rows
    [row0, row0 + rows), as a local CSR (rowptr from 0)."""
    rank: int
    t0: int
    t1: int
    rows: int
    n: int
    rowptr: np.ndarray
    colidx: np.ndarray
    val: np.ndarray
    products: int
    row0: int = 0
    nnz0: int = 0
    nnz_total: int = 0
    per_rank: list = field(default_factory=list)

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1]) if self.rowptr.size else 0


def plan(matA, matB, world: int):
    """(per-tile-row scalar products of A*B, the world's tile-row ranges)."""
    tile_prods = blocks.tile_row_products(matA, matB)
    return tile_prods, blocks.partition(tile_prods, world)


def compute_piece(matA, matB, rank: int, world: int, multiply, budget: float = 1.5e9) -> Piece:
    """Rank `rank`'s piece of C = A*B.  `multiply(block_csr_of_A, matB)`
    returns the block's C as (rowptr, colidx, val) host arrays (the device
    product in use; any exact multiply in a test); blocks within the range
    hold at most `budget` scalar products each."""
    tile_prods, ranges = plan(matA, matB, world)
    t0, t1 = ranges[rank]
    m = matA[0]
    rows = min(t1 * blocks.TILE, m) - min(t0 * blocks.TILE, m)
    rp_parts, ci_parts, v_parts, base = [np.zeros(1, np.int64)], [], [], 0
    for b0, b1 in blocks.row_blocks(tile_prods[t0:t1], budget):
        rp, ci, v = multiply(blocks.block_rows(matA, t0 + b0, t0 + b1), matB)
        rp = np.asarray(rp, np.int64)
        rp_parts.append(rp[1:] + base)
        ci_parts.append(np.asarray(ci))
        v_parts.append(np.asarray(v))
        base += int(rp[-1])
    rowptr = np.concatenate(rp_parts)
    assert rowptr.size == rows + 1, "blocks do not cover the range's rows"
    return Piece(rank, t0, t1, rows, matB[1], rowptr,
                 np.concatenate(ci_parts) if ci_parts else np.zeros(0, np.int32),
                 np.concatenate(v_parts) if v_parts else np.zeros(0, np.float64),
                 int(tile_prods[t0:t1].sum()))


def global_offsets(rows: int, nnz: int, dist=None, device="cpu"):
    """All-gather of every rank's (rows, nnz): returns (row0, nnz0, total
    nnz, [(rows, nnz) per rank]) for this rank.  Without a process group the
    caller is the only rank."""
    if dist is None:
        return 0, 0, nnz, [(rows, nnz)]
    import torch
    mine = torch.tensor([rows, nnz], dtype=torch.int64, device=device)
    allv = [torch.zeros(2, dtype=torch.int64, device=device) for _ in range(dist.get_world_size())]
    dist.all_gather(allv, mine)
    per = [(int(t[0]), int(t[1])) for t in allv]
    r = dist.get_rank()
    return (sum(p[0] for p in per[:r]), sum(p[1] for p in per[:r]), sum(p[1] for p in per), per)


def place(piece: Piece, dist=None, device="cpu") -> Piece:
    """Fills the piece's global offsets (the all-gather)."""
    piece.row0, piece.nnz0, piece.nnz_total, piece.per_rank = global_offsets(piece.rows, piece.nnz, dist, device)
    return piece


def assemble(pieces) -> tuple:
    """The whole CSR of C from every rank's piece (in rank order), for a
    consumer that gathers it on one host."""
    pieces = sorted(pieces, key=lambda p: p.rank)
    rp, base = [np.zeros(1, np.int64)], 0
    for p in pieces:
        rp.append(p.rowptr[1:] + base)
        base += p.nnz
    m = sum(p.rows for p in pieces)
    n = pieces[0].n if pieces else 0
    return (m, n, np.concatenate(rp), np.concatenate([p.colidx for p in pieces]),
            np.concatenate([p.val for p in pieces]))
