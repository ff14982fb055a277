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


def from_extents(ext: np.ndarray, bc: Sequence[int], h: Sequence[float], ngrid: int, pl: int = 1):
    """Descriptors for blocks with integer extents ext[b] = (xs, xe, ys, ye, zs, ze)."""
    ext = np.ascontiguousarray(ext, dtype=np.int32).reshape(-1, 6)
    nb = ext.shape[0]
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
               pl: int = 1):
    """A regular nblk[0] x nblk[1] x nblk[2] arrangement of equal blocks of n cells.

    Blocks are numbered x fastest (as the reference's type-2 infodom layout,
    alloc_dom.for:466-477)."""
    ext = []
    for k in range(nblk[2]):
        for j in range(nblk[1]):
            for i in range(nblk[0]):
                ext.append((i * n[0], (i + 1) * n[0], j * n[1], (j + 1) * n[1], k * n[2], (k + 1) * n[2]))
    return from_extents(np.array(ext), bc, h, ngrid, pl)


def independent_blocks(sizes: Sequence[Sequence[int]], h: Sequence[float], ngrid: int, pl: int = 1):
    """Blocks that do not touch (each an isolated all-wall Poisson problem)."""
    ext = []
    x = 0
    for s in sizes:
        ext.append((x, x + s[0], 0, s[1], 0, s[2]))
        x += s[0] + 1  # a one-cell gap: no face, edge or corner contact
    return from_extents(np.array(ext), [WALL] * 6, h, ngrid, pl)
