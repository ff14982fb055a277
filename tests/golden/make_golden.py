"""Write the golden mgkcyc fixtures of tests/golden/ from the reference's own Fortran.

    python tests/golden/make_golden.py        (needs the reference source tree)

Each fixture runs the reference's coeff + mgkcyc (mgsolver.for:2-372 with
mgrelax/mgrestr/mgcorr/mgbound and exchangepp/exchbc_mgpp from
exchangepp.for), translated statement by statement by oracle/fortran_ref.py,
on one block layout with seeded random inputs, and stores the inputs and the
resulting pressure correction pp.  Ghost layers beyond the first one, which
the multigrid path must never read, are filled with NaN in the reference run.

Stored per block (x fastest, one ghost layer): pp_in, pp_out (nz+2, ny+2,
nx+2), su (nz, ny, nx) and, for L_LSM cases, dens (nz, ny, nx).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import fortran_ref as F  # noqa: E402
from oracle import oracle as O  # noqa: E402

W, P = 4, 5

# The reference's Fortran sources: H3D_REFERENCE_SRC if set, else the
# read-only mount of the reference tree this script was written against.
REF_SRC = F.REF_SRC or "/root/reference/src_v70"


def grid(nb, n):
    ext = []
    for k in range(nb[2]):
        for j in range(nb[1]):
            for i in range(nb[0]):
                ext.append((i * n[0], (i + 1) * n[0], j * n[1], (j + 1) * n[1], k * n[2], (k + 1) * n[2]))
    return np.array(ext, dtype=np.int32)


# name: (layout, bc, ngrd_gl, mg_itrsch, pl_ex, lsm, seed)
CASES = {
    "walls_2x1x1": (grid((2, 1, 1), (8, 8, 8)), [W] * 6, 3, 3, 0, False, 101),
    "periodic_x_2x2x2": (grid((2, 2, 2), (8, 8, 8)), [P, P, W, W, W, W], 3, 3, 2, False, 102),
    "periodic_all_2x1x3": (grid((2, 1, 3), (8, 8, 8)), [P] * 6, 3, 3, 0, False, 103),
    "periodic_y_noncubic_3x2x1": (grid((3, 2, 1), (16, 8, 8)), [W, W, P, P, W, W], 3, 3, 0, False, 104),
    "lsm_periodic_x_2x1x2": (grid((2, 1, 2), (8, 8, 8)), [P, P, W, W, W, W], 3, 3, 0, True, 105),
    "lexgs_2x2x1": (grid((2, 2, 1), (8, 8, 8)), [W, W, P, P, W, W], 3, 1, 0, False, 106),
    "tdma_2x2x1": (grid((2, 2, 1), (8, 8, 8)), [W] * 6, 3, 2, 0, False, 107),
}
H = (1.0 / 32, 1.0 / 32, 1.0 / 32)


def run_case(name, src_dir=REF_SRC):
    ext, bc, ngrd, itr, pl_ex, lsm, seed = CASES[name]
    descs = O.topology(ext, bc, H, ngrd)
    R = F.Reference(list(descs), ngrd, mg_itrsch=itr, pl_ex=pl_ex, lsm=lsm, src_dir=src_dir)
    pl = R.pl
    rng = np.random.default_rng(seed)
    out = {"ext": ext, "bc": np.array(bc, np.int32), "h": np.array(H), "ngrd_gl": ngrd, "mg_itrsch": itr,
           "pl": pl, "lsm": int(lsm), "nblocks": len(descs)}
    for ib, d in enumerate(descs):
        nx, ny, nz = d.n
        shp = (nz + 2 * pl, ny + 2 * pl, nx + 2 * pl)
        pp_in = rng.standard_normal((nz + 2, ny + 2, nx + 2))
        su = rng.standard_normal((nz, ny, nx))
        full = np.full(shp, np.nan)
        full[pl - 1:pl + nz + 1, pl - 1:pl + ny + 1, pl - 1:pl + nx + 1] = pp_in
        R.put_field("pp", ib, full)
        full = np.full(shp, np.nan)
        full[pl:pl + nz, pl:pl + ny, pl:pl + nx] = su
        R.put_field("su", ib, full)
        R.put_field("sup", ib, full)
        out["pp_in_%d" % ib] = pp_in
        out["su_%d" % ib] = su
        if lsm:
            dens = 1.0 + 999.0 * rng.random((nz, ny, nx))
            full = np.full(shp, np.nan)
            full[pl:pl + nz, pl:pl + ny, pl:pl + nx] = dens
            R.put_field("dens", ib, full)
            out["dens_%d" % ib] = dens
    R.call("coeff")
    R.call("mgkcyc")
    for ib, d in enumerate(descs):
        nx, ny, nz = d.n
        pp = R.get_field("pp", ib)
        out["pp_out_%d" % ib] = pp[pl - 1:pl + nz + 1, pl - 1:pl + ny + 1, pl - 1:pl + nx + 1].copy()
        if not np.isfinite(out["pp_out_%d" % ib]).all():
            raise RuntimeError("%s: the reference produced non-finite values" % name)
    return out


def main():
    for name in CASES:
        data = run_case(name)
        np.savez_compressed(os.path.join(HERE, "mgkcyc_%s.npz" % name), **data)
        print("wrote", name)


if __name__ == "__main__":
    main()
