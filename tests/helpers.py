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


def projection_fields(blocks, seed, lsm=False, dens_hi=1000.0):
    """Seeded canonical per-block inputs of the projection (newsolv_mg with
    velocities): p, u, v, w, ustar, vstar, wstar (and a density for L_LSM),
    each (nz+2, ny+2, nx+2), x fastest.

    Everything is random (ghosts included) except the velocity faces on
    physical walls, which are zero, so the pressure equation is compatible
    (the density, L_LSM only, is uniform in [1, dens_hi]):
    u at x = 0 of a block whose west face is a wall and at x = nx when the east
    face is, and likewise v and w."""
    rng = np.random.default_rng(seed)
    out = {k: [] for k in ("p", "u", "v", "w", "us", "vs", "ws", "dens")}
    for d in blocks:
        shp = (d.n[2] + 2, d.n[1] + 2, d.n[0] + 2)
        for k in ("p", "us", "vs", "ws"):
            out[k].append(rng.uniform(-1.0, 1.0, shp))
        for ax, k in enumerate(("u", "v", "w")):
            a = rng.uniform(-1.0, 1.0, shp)
            lo = d.nb_face[2 * ax] < 0 and d.bc[2 * ax] != 5
            hi = d.nb_face[2 * ax + 1] < 0 and d.bc[2 * ax + 1] != 5
            idx_lo = [slice(None)] * 3
            idx_hi = [slice(None)] * 3
            idx_lo[2 - ax] = 0
            idx_hi[2 - ax] = d.n[ax]
            if lo:
                a[tuple(idx_lo)] = 0.0
            if hi:
                a[tuple(idx_hi)] = 0.0
            out[k].append(a)
        out["dens"].append(rng.uniform(1.0, dens_hi, shp) if lsm else np.ones(shp))
    return out


def to_host(blocks, canon):
    """Canonical per-block arrays -> host fields (ttc dims, pl ghosts)."""
    res = []
    for a, d in zip(canon, blocks):
        h = np.zeros((d.ttc[2], d.ttc[1], d.ttc[0]))
        p = d.pl
        h[p - 1:p + d.n[2] + 1, p - 1:p + d.n[1] + 1, p - 1:p + d.n[0] + 1] = a
        res.append(h)
    return res


def apply_expr(nodes, dst, src, flat):
    """Applies an expression fill (h3d_halo_expr) to the concatenated
    canonical arrays `flat` in place, in FP64 with the operation order the
    table states.  Pre-fill values are those of `flat` on entry."""
    flat = np.asarray(flat)
    old = flat.copy()
    vals = np.zeros(len(nodes))

    def ref(r):
        r = np.asarray(r, dtype=np.uint32)
        tag = r >> np.uint32(30)
        idx = (r & np.uint32(0x3FFFFFFF)).astype(np.int64)
        out = np.zeros(r.shape)
        m = tag == 0
        out[m] = flat[idx[m]]
        m = tag == 1
        out[m] = vals[idx[m]]
        m = tag == 2
        out[m] = old[idx[m]]
        return out

    if len(nodes):
        op = nodes[:, 0]
        # operands name lower-index nodes only: evaluate until nothing changes
        # (one pass per depth)
        depth = np.zeros(len(nodes), dtype=np.int64)
        for k in range(len(nodes)):
            for q in range(1, 9):
                r = int(nodes[k, q])
                if r >> 30 == 1:
                    depth[k] = max(depth[k], depth[r & 0x3FFFFFFF] + 1)
        for d in range(int(depth.max()) + 1):
            sel = np.nonzero(depth == d)[0]
            a = [ref(nodes[sel, q]) for q in range(1, 9)]
            o = op[sel]
            v = np.zeros(len(sel))
            m = o == 0
            v[m] = a[0][m]
            m = o == 1
            s = a[0][m]
            for q in range(1, 8):
                s = s + a[q][m]
            v[m] = s * 0.125
            m = o == 2
            v[m] = 2.0 * a[0][m]
            m = o == 3
            v[m] = ((a[0][m] + 3.0 * a[1][m]) - a[2][m]) / 4.0
            m = o == 4
            w = (27.0, 9.0, 9.0, 3.0, 9.0, 3.0, 3.0, 1.0)
            s = w[0] * a[0][m]
            for q in range(1, 8):
                s = s + w[q] * a[q][m]
            v[m] = s / 64.0
            vals[sel] = v
    flat[np.asarray(dst, dtype=np.int64)] = ref(src)
    return flat
