"""Block sharding of a multi-block level across ranks (one GPU per rank).

The reference runs its blocks on MPI ranks and fills the ghosts of a level
with exchangepp (src_v70/exchangepp.for:2-2835): same-rank neighbours are
packed straight into the receiver's buffer, other ranks' by MPI_SEND /
MPI_IRECV (:423-428 for the faces, :1382-1387 for corners and edges), and
the norms go through MPI_ALLREDUCE (newsolv_mg.for:33, press.for:72).
Here the exchange is resolved once, on cell identities, into the gather
table of h3d_halo_table (every ghost cell -> the one cell whose value it
ends up holding); sharding splits that table by owner:

  * entries whose source and destination blocks live on this rank are a
    local gather (the single-GPU fill kernel);
  * entries whose source lives on rank r become one packed message r -> this
    rank per fill, in table order on both sides, so no index travels at run
    time: the sender gathers its values into a contiguous buffer, the
    receiver scatters the buffer into its ghost cells.

One fill is one grouped point-to-point round: every rank posts its receives
and sends to every peer it shares a face, edge or corner with (NCCL grouped
send/recv of device buffers between GPUs; torch.distributed over gloo for the
CPU tests).  Norms are reduced deterministically: each rank contributes its
blocks' partial sums, every rank gathers all of them and adds them in block
order, so the result is the single-rank one bit for bit.

Layout of a rank's level array: its own blocks, in block order, each the
canonical (nz+2, ny+2, nx+2) array x fastest (the numbering h3d_halo_table
uses, restricted to the owned blocks).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Sequence

import numpy as np

IDX_MASK = 0x7FFFFFFF


def partition(blocks: Sequence, world: int) -> List[int]:
    """Owner rank of every block: contiguous runs of blocks (block order, the
    reference's rank assignment in mdmap order) with about equal cell counts."""
    cells = np.array([d.n[0] * d.n[1] * d.n[2] for d in blocks], dtype=np.float64)
    total = cells.sum()
    owner, r, acc = [], 0, 0.0
    for c in cells:
        # move to the next rank once this one holds its share
        if r < world - 1 and acc >= total * (r + 1) / world:
            r += 1
        owner.append(r)
        acc += c
    return owner


def _level_sizes(blocks, g):
    s = 2 ** (g - 1)
    return [(d.n[0] // s + 2) * (d.n[1] // s + 2) * (d.n[2] // s + 2) for d in blocks]


@dataclass
class HaloPlan:
    """The ghost fill of level g split for one rank."""

    rank: int
    owner: List[int]
    local_dst: np.ndarray = None
    local_src: np.ndarray = None
    send_idx: Dict[int, np.ndarray] = field(default_factory=dict)  # peer -> local source cells
    recv_idx: Dict[int, np.ndarray] = field(default_factory=dict)  # peer -> local ghost cells
    n_local_cells: int = 0


def build_plan(blocks: Sequence, g: int, kind: int, owner: Sequence[int], rank: int, table=None) -> HaloPlan:
    """Split the gather table of level g (h3d_halo_table kind) for `rank`.
    `table` = (dst, src) in the global packed numbering, else it is built by
    the library (host-only, no GPU)."""
    if table is None:
        from .mg import halo_table
        table = halo_table(blocks, g, kind)
    dst, src = (np.asarray(a, dtype=np.int64) for a in table)
    src = src & IDX_MASK  # old / current value: both read the pre-fill snapshot here
    sizes = _level_sizes(blocks, g)
    starts = np.concatenate([[0], np.cumsum(sizes)])
    blk_dst = np.searchsorted(starts, dst, side="right") - 1
    blk_src = np.searchsorted(starts, src, side="right") - 1
    own = np.asarray(owner)
    # global -> local numbering of every rank
    local_start = {}
    for r in set(owner):
        off = 0
        for b, o in enumerate(owner):
            if o == r:
                local_start[b] = off
                off += sizes[b]
    def to_local(idx, blk):
        return np.array([local_start[b] for b in blk], dtype=np.int64) + (idx - starts[blk])
    od, os_ = own[blk_dst], own[blk_src]
    plan = HaloPlan(rank=rank, owner=list(owner))
    plan.n_local_cells = int(sum(sizes[b] for b, o in enumerate(owner) if o == rank))
    m = (od == rank) & (os_ == rank)
    plan.local_dst = to_local(dst[m], blk_dst[m])
    plan.local_src = to_local(src[m], blk_src[m])
    for peer in sorted(set(owner)):
        if peer == rank:
            continue
        ms = (os_ == rank) & (od == peer)   # this rank's cells another rank needs
        mr = (od == rank) & (os_ == peer)   # this rank's ghosts another rank fills
        if ms.any():
            plan.send_idx[peer] = to_local(src[ms], blk_src[ms])
        if mr.any():
            plan.recv_idx[peer] = to_local(dst[mr], blk_dst[mr])
    return plan


def exchange(plan: HaloPlan, level: np.ndarray, dist=None) -> np.ndarray:
    """One ghost fill of this rank's level array (in place; returned).  All
    values are read from the pre-fill snapshot, as the single-GPU gather does.
    `dist` is torch.distributed (None: one rank)."""
    snap = level.copy()
    if plan.send_idx or plan.recv_idx:
        import torch
        reqs, bufs = [], {}
        for peer, idx in plan.recv_idx.items():
            bufs[peer] = torch.empty(len(idx), dtype=torch.float64)
            reqs.append(dist.irecv(bufs[peer], src=peer))
        for peer, idx in plan.send_idx.items():
            reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(snap[idx])), dst=peer))
        for q in reqs:
            q.wait()
    level[plan.local_dst] = snap[plan.local_src]
    for peer, idx in plan.recv_idx.items():
        level[idx] = bufs[peer].numpy()
    return level


def reduce_block_sums(per_block: Dict[int, np.ndarray], nblocks: int, dist=None) -> np.ndarray:
    """Sum of per-block partial sums (each a vector), added in block order on
    every rank: the single-rank result bit for bit."""
    width = len(next(iter(per_block.values()))) if per_block else 0
    mine = np.full((nblocks, width + 1), np.nan)
    mine[:, 0] = 0.0
    for b, v in per_block.items():
        mine[b, 0] = 1.0
        mine[b, 1:] = v
    if dist is not None:
        import torch
        world = dist.get_world_size()
        parts = [torch.empty(mine.shape, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(parts, torch.from_numpy(mine))
        rows = np.full((nblocks, width), np.nan)
        for p in parts:
            a = p.numpy()
            sel = a[:, 0] == 1.0
            rows[sel] = a[sel, 1:]
    else:
        rows = mine[:, 1:]
    total = np.zeros(rows.shape[1])
    for b in range(nblocks):
        total = total + rows[b]
    return total
