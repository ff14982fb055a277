"""Shared helpers of the test-suite (oracle <-> product plumbing)."""
import ctypes as C

import numpy as np


def to_oracle_descs(O, blocks):
    """Product h3d_block_desc list -> oracle or_block_desc list (same bytes)."""
    od = (O.BlockDesc * len(blocks))()
    src = (type(blocks[0]) * len(blocks))(*blocks)
    C.memmove(od, src, C.sizeof(od))
    return list(od)


def canon_from_host(a, d):
    """Host field (ttc, pl ghosts) -> canonical (n+2)^3 with one ghost layer."""
    p = d.pl
    return np.ascontiguousarray(a[p - 1:p + d.n[2] + 1, p - 1:p + d.n[1] + 1, p - 1:p + d.n[0] + 1])


def interior_of_host(a, d):
    p = d.pl
    return np.ascontiguousarray(a[p:p + d.n[2], p:p + d.n[1], p:p + d.n[0]])


def mean_removed_rel(a, b):
    """Relative L2 difference after removing each field's mean."""
    a = np.concatenate([x.ravel() for x in a])
    b = np.concatenate([x.ravel() for x in b])
    a = a - a.mean()
    b = b - b.mean()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
