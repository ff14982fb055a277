"""Block layouts of the multi-block domain (the `multidom` descriptors).

Neighbour discovery is the library's restatement of read_infodom
(src_v70/alloc_dom.for:524-1200) on integer block extents.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib

WALL = 4       # any bc code other than 5 is a zero-gradient wall for p
PERIODIC = 5   # control.cin periodic code


def grid_extents(nblk: Sequence[int], n: Sequence[int]) -> np.ndarray:
    """Extents of a regular nblk[0] x nblk[1] x nblk[2] arrangement of equal
    blocks of n cells, numbered x fastest (the reference's type-2 infodom
    layout, alloc_dom.for:466-477)."""
    ext = []
    for k in range(nblk[2]):
        for j in range(nblk[1]):
            for i in range(nblk[0]):
                ext.append((i * n[0], (i + 1) * n[0], j * n[1], (j + 1) * n[1], k * n[2], (k + 1) * n[2]))
    return np.array(ext, dtype=np.int32)


def gap_extents(sizes: Sequence[Sequence[int]]) -> np.ndarray:
    """Extents of blocks laid out along x with a one-cell gap between
    neighbours, so no two blocks share a face, edge or corner."""
    ext = []
    x = 0
    for s in sizes:
        ext.append((x, x + s[0], 0, s[1], 0, s[2]))
        x += s[0] + 1
    return np.array(ext, dtype=np.int32)


def from_extents(ext: np.ndarray, bc: Sequence[int], h: Sequence[float], ngrid: int, pl: int = 1,
                 resolve=None):
    """Descriptors for blocks with integer extents ext[b] = (xs, xe, ys, ye, zs, ze).

    Neighbours are found by the library's h3d_topology; `resolve(ext, bc, h,
    ngrid)`, if given, is called instead and must return descriptors with the
    h3d_block_desc layout."""
    ext = np.ascontiguousarray(ext, dtype=np.int32).reshape(-1, 6)
    nb = ext.shape[0]
    if resolve is not None:
        out = resolve(ext, bc, h, ngrid)
        for d in out:
            d.pl = pl
            for a in range(3):
                d.ttc[a] = d.n[a] + 2 * pl
        return list(out)
    bcv = np.ascontiguousarray(bc, dtype=np.int32)
    hv = np.ascontiguousarray(h, dtype=np.float64)
    out = (_lib.BlockDesc * nb)()
    rc = _lib.lib().h3d_topology(nb, ext.ctypes.data_as(C.POINTER(C.c_int32)),
                                 bcv.ctypes.data_as(C.POINTER(C.c_int32)),
                                 hv.ctypes.data_as(C.POINTER(C.c_double)), int(ngrid), out)
    _lib.check(rc, None, "h3d_topology")
    for d in out:
        d.pl = pl
        for a in range(3):
            d.ttc[a] = d.n[a] + 2 * pl
    return list(out)


def block_grid(nblk: Sequence[int], n: Sequence[int], bc: Sequence[int], h: Sequence[float], ngrid: int,
               pl: int = 1, resolve=None):
    """A regular nblk[0] x nblk[1] x nblk[2] arrangement of equal blocks of n
    cells, numbered x fastest (alloc_dom.for:466-477)."""
    return from_extents(grid_extents(nblk, n), bc, h, ngrid, pl, resolve)


def independent_blocks(sizes: Sequence[Sequence[int]], h: Sequence[float], ngrid: int, pl: int = 1,
                       resolve=None):
    """Blocks that do not touch (each an isolated all-wall Poisson problem)."""
    return from_extents(gap_extents(sizes), [WALL] * 6, h, ngrid, pl, resolve)


def refine(descs, rdiv: Sequence[int], ngrid_input: int):
    """Local mesh refinement of a layout (LMR = 2, localparameters.for:24-59,
    102-104, 247-249): block b keeps its physical extent and gets rdiv[b]
    times the cells per axis, spacing h / rdiv[b] and ngrid_input +
    log2(rdiv[b]) levels.  `descs` are the unrefined descriptors (ngrid and h
    of the coarse layout); they are changed in place and returned.  Face,
    edge and corner neighbours may differ by a factor of 2 in rdiv."""
    for d, r in zip(descs, rdiv):
        r = int(r)
        lg = r.bit_length() - 1
        if r < 1 or (1 << lg) != r:
            raise ValueError("rdiv must be a power of 2")
        for a in range(3):
            d.n[a] = d.n[a] * r
            d.h[a] = d.h[a] / r
            d.origin[a] = d.origin[a] * r
            d.ttc[a] = d.n[a] + 2 * d.pl
        d.rdiv = r
        d.ngrid = int(ngrid_input) + lg
    return descs
