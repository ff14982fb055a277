"""Write the golden fixtures of tests/golden/ from the reference's own Fortran.

    python tests/golden/make_golden.py        (needs the reference source tree)

Each fixture runs the reference's coeff + mgkcyc (mgsolver.for:2-372 with
mgrelax/mgrestr/mgcorr/mgbound and exchangepp/exchbc_mgpp from
exchangepp.for), translated statement by statement by oracle/fortran_ref.py,
on one block layout with seeded random inputs, and stores the inputs and the
resulting pressure correction pp.  Ghost layers beyond the first one, which
the multigrid path must never read, are filled with NaN in the reference run.

Stored per block (x fastest, one ghost layer): pp_in, pp_out (nz+2, ny+2,
nx+2), su (nz, ny, nx) and, for L_LSM cases, dens (nz, ny, nx).

The project_*.npz fixtures run the reference's calvel, calmas, mgkcyc,
exchange(4) and pbound (press.for, exchange.for, exchange_bc.for) in the
order of newsolv_mg's loop; see run_projection_case.  The sip_*.npz fixtures
run the SIP pressure path (sipsol.for and press.for's pressure_1sweep loop);
see run_sip_case.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import fortran_ref as F  # noqa: E402
from oracle import oracle as O  # noqa: E402
from hydro3d_b200.topology import refine  # noqa: E402

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
# Local mesh refinement (LMR = 2): the layout above is the unrefined one and its
# ngrd_gl is ngrid_input; block b gets rdiv[b] (hydro3d_b200.topology.refine).
# Periodic partners keep equal ratios (exchbc_mgpp has no refinement branch).
LMR_CASES = {
    "lmr_walls_2x1x1": (grid((2, 1, 1), (8, 8, 8)), [W] * 6, 3, 3, 0, False, 111, [1, 2]),
    "lmr_corners_2x2x2": (grid((2, 2, 2), (8, 8, 8)), [W] * 6, 3, 3, 0, False, 112, [2, 1, 1, 1, 1, 1, 1, 1]),
    "lmr_periodic_x_1x2x2": (grid((1, 2, 2), (8, 8, 8)), [P, P, W, W, W, W], 2, 3, 0, False, 113, [1, 2, 2, 1]),
    "lmr_ratio4_2x2x1": (grid((2, 2, 1), (4, 4, 4)), [W, W, W, W, P, P], 2, 3, 0, False, 114, [2, 2, 2, 4]),
    "lmr_tdma_2x2x1": (grid((2, 2, 1), (8, 8, 8)), [W] * 6, 3, 2, 0, False, 115, [1, 2, 2, 1]),
}
CASES.update(LMR_CASES)
H = (1.0 / 32, 1.0 / 32, 1.0 / 32)


def lmr_descs(ext, bc, h, ngrid_input, rdiv):
    """The unrefined layout's descriptors, refined by rdiv, and ngrd_gl."""
    descs = refine(list(O.topology(ext, bc, h, ngrid_input)), rdiv, ngrid_input)
    return descs, ngrid_input + max(int(r).bit_length() - 1 for r in rdiv)


def run_case(name, src_dir=REF_SRC):
    ext, bc, ngrd, itr, pl_ex, lsm, seed = CASES[name][:7]
    rdiv = CASES[name][7] if len(CASES[name]) > 7 else None
    if rdiv is None:
        descs = O.topology(ext, bc, H, ngrd)
    else:
        descs, ngrd = lmr_descs(ext, bc, H, ngrd, rdiv)
    R = F.Reference(list(descs), ngrd, mg_itrsch=itr, pl_ex=pl_ex, lsm=lsm, src_dir=src_dir)
    pl = R.pl
    rng = np.random.default_rng(seed)
    out = {"ext": ext, "bc": np.array(bc, np.int32), "h": np.array(H), "ngrd_gl": ngrd, "mg_itrsch": itr,
           "pl": pl, "lsm": int(lsm), "nblocks": len(descs)}
    if rdiv is not None:
        out["rdiv"] = np.array(rdiv, np.int32)
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


# The projection (newsolv_mg with the velocities): name -> (layout, bc, ngrd_gl, lsm, seed)
PROJ_CASES = {
    "walls_2x1x1": (grid((2, 1, 1), (8, 8, 8)), [W] * 6, 3, False, 201),
    "periodic_x_2x2x1": (grid((2, 2, 1), (8, 8, 8)), [P, P, W, W, W, W], 3, False, 202),
    "periodic_all_1x2x2": (grid((1, 2, 2), (8, 8, 8)), [P] * 6, 3, False, 203),
    "lsm_periodic_y_2x2x1": (grid((2, 2, 1), (8, 8, 8)), [W, W, P, P, W, W], 3, True, 204),
}
DT, ALFAPR, NITER = 0.5, 0.9, 2


def run_projection_case(name, src_dir=REF_SRC):
    """The reference's own calvel (with its exchange(1..3)), calmas, mgkcyc,
    exchange(4) and pbound in newsolv_mg's order (newsolv_mg.for:16-55),
    NITER iterations from seeded p, u, v, w, ustar, vstar, wstar (wall faces
    of u, v, w zero), pl = 1 so the host arrays are the canonical ones.
    Stored per block: the inputs, and after the loop p, u, v, w, su (sup for
    L_LSM) and the rmax after the first calmas and after every iteration."""
    ext, bc, ngrd, lsm, seed = PROJ_CASES[name]
    descs = O.topology(ext, bc, H, ngrd)
    R = F.Reference(list(descs), ngrd, pl_ex=0, lsm=lsm, src_dir=src_dir)
    M = R.M
    M.v_rdivmax = 1        # alloc_dom.for: the largest rdiv (no refinement)
    M.v_differencing = 1   # second-order branch of calmas (press.for:40-58)
    M.v_dt = DT
    M.v_alfapr = ALFAPR
    assert R.pl == 1
    rng = np.random.default_rng(seed)
    out = {"ext": ext, "bc": np.array(bc, np.int32), "h": np.array(H), "ngrd_gl": ngrd, "lsm": int(lsm),
           "nblocks": len(descs), "dt": DT, "alfapr": ALFAPR, "niter": NITER}
    for ib, d in enumerate(descs):
        nx, ny, nz = d.n
        shp = (nz + 2, ny + 2, nx + 2)
        for k in ("p", "ustar", "vstar", "wstar"):
            a = rng.uniform(-1.0, 1.0, shp)
            R.put_field(k, ib, a)
            out["%s_in_%d" % (k, ib)] = a
        for ax, k in enumerate(("u", "v", "w")):
            a = rng.uniform(-1.0, 1.0, shp)
            lo = d.nb_face[2 * ax] < 0 and d.bc[2 * ax] != 5
            hi = d.nb_face[2 * ax + 1] < 0 and d.bc[2 * ax + 1] != 5
            sl = [slice(None)] * 3
            if lo:
                sl[2 - ax] = 0
                a[tuple(sl)] = 0.0
            if hi:
                sl[2 - ax] = d.n[ax]
                a[tuple(sl)] = 0.0
            R.put_field(k, ib, a)
            out["%s_in_%d" % (k, ib)] = a
        if lsm:
            dens = rng.uniform(1.0, 4.0, shp)
            R.put_field("dens", ib, dens)
            out["dens_%d" % ib] = dens
        R.put_field("pp", ib, np.zeros(shp))
    R.call("coeff")
    rmax = []
    R.call("calvel")
    R.call("calmas")
    rmax.append(M.v_rmax)
    for _ in range(NITER):
        R.call("mgkcyc")
        for ib in range(len(descs)):  # newsolv_mg.for:39-49 (ppref = 0)
            p = R.get_field("p", ib)
            pp = R.get_field("pp", ib)
            R.put_field("p", ib, p + (pp - 0.0))
            R.put_field("pp", ib, np.zeros_like(pp))
        R.call("exchange", 4)
        R.call("pbound")
        R.call("calvel")
        R.call("calmas")
        rmax.append(M.v_rmax)
    out["rmax"] = np.array(rmax)
    for ib in range(len(descs)):
        for k in ("p", "u", "v", "w"):
            out["%s_out_%d" % (k, ib)] = R.get_field(k, ib)
        s = R.get_field("sup" if lsm else "su", ib)
        out["su_out_%d" % ib] = s[1:-1, 1:-1, 1:-1].copy()
        for k in ("p_out", "u_out", "su_out"):
            if not np.isfinite(out["%s_%d" % (k, ib)]).all():
                raise RuntimeError("%s: the reference produced non-finite values" % name)
    return out


# The SIP pressure path (solver = 1): name -> (layout, bc, nswp, seed)
SIP_CASES = {
    "walls_2x1x1": (grid((2, 1, 1), (8, 8, 8)), [W] * 6, 6, 301),
    "periodic_x_2x2x1": (grid((2, 2, 1), (8, 8, 8)), [P, P, W, W, W, W], 60, 302),
    "periodic_all_1x2x2": (grid((1, 2, 2), (8, 8, 8)), [P] * 6, 60, 303),
}
SIP_NITER = 2


def run_sip_case(name, src_dir=REF_SRC):
    """The reference's pressure_1sweep loop (press.for:439-472) from its own
    calvel, calmas, sipsol(44), exchange(4) and pbound, SIP_NITER iterations
    of at most nswp sweeps, with the coefficients pressure_1sweep builds
    (press.for:407-438, restated below in its loop order and operand order).
    Stored per block: the inputs, p, u, v, w and pp after the loop, the rmax
    of every calmas and the sweep count of every sipsol."""
    ext, bc, nswp, seed = SIP_CASES[name]
    descs = O.topology(ext, bc, H, 2)
    R = F.Reference(list(descs), 2, pl_ex=0, lsm=False, src_dir=src_dir)
    M = R.M
    M.v_rdivmax = 1
    M.v_differencing = 1
    M.v_dt = DT
    M.v_alfapr = ALFAPR
    M.v_nswp = F.FArray("i", [(1, 4)])
    M.v_nswp.fill(nswp)
    rng = np.random.default_rng(seed)
    out = {"ext": ext, "bc": np.array(bc, np.int32), "h": np.array(H), "nblocks": len(descs), "dt": DT,
           "alfapr": ALFAPR, "nswp": nswp, "niter": SIP_NITER}
    for ib, d in enumerate(descs):
        nx, ny, nz = d.n
        shp = (nz + 2, ny + 2, nx + 2)
        for k in ("p", "ustar", "vstar", "wstar"):
            a = rng.uniform(-1.0, 1.0, shp)
            R.put_field(k, ib, a)
            out["%s_in_%d" % (k, ib)] = a
        for ax, k in enumerate(("u", "v", "w")):
            a = rng.uniform(-1.0, 1.0, shp)
            sl = [slice(None)] * 3
            if d.nb_face[2 * ax] < 0 and d.bc[2 * ax] != 5:
                sl[2 - ax] = 0
                a[tuple(sl)] = 0.0
            if d.nb_face[2 * ax + 1] < 0 and d.bc[2 * ax + 1] != 5:
                sl[2 - ax] = d.n[ax]
                a[tuple(sl)] = 0.0
            R.put_field(k, ib, a)
            out["%s_in_%d" % (k, ib)] = a
        # press.for:401-438: ap, pp, su zeroed, then the coefficients
        o = R.dom(ib)
        dx, dy, dz = o.c_dx, o.c_dy, o.c_dz
        co = {k: np.zeros(shp) for k in ("aw", "ae", "an", "as", "at", "ab", "ap")}
        for k in range(1, nz + 1):
            for i in range(1, nx + 1):
                for j in range(1, ny + 1):
                    co["aw"][k, j, i] = 1.0 / (dx * dx)
                    co["ae"][k, j, i] = 1.0 / (dx * dx)
                    co["an"][k, j, i] = 1.0 / (dy * dy)
                    co["as"][k, j, i] = 1.0 / (dy * dy)
                    co["at"][k, j, i] = 1.0 / (dz * dz)
                    co["ab"][k, j, i] = 1.0 / (dz * dz)
                    if d.nb_face[0] < 0 and d.bc[0] != 5:
                        co["aw"][k, j, 1] = 0.0
                    if d.nb_face[1] < 0 and d.bc[1] != 5:
                        co["ae"][k, j, nx] = 0.0
                    if d.nb_face[2] < 0 and d.bc[2] != 5:
                        co["as"][k, 1, i] = 0.0
                    if d.nb_face[3] < 0 and d.bc[3] != 5:
                        co["an"][k, ny, i] = 0.0
                    if d.nb_face[4] < 0 and d.bc[4] != 5:
                        co["ab"][1, j, i] = 0.0
                    if d.nb_face[5] < 0 and d.bc[5] != 5:
                        co["at"][nz, j, i] = 0.0
                    co["ap"][k, j, i] = -1.0 * (co["aw"][k, j, i] + co["ae"][k, j, i] + co["as"][k, j, i] +
                                                co["an"][k, j, i] + co["ab"][k, j, i] + co["at"][k, j, i])
        for k2, a in co.items():
            R.put_field(k2, ib, a)
        R.put_field("pp", ib, np.zeros(shp))
        R.put_field("su", ib, np.zeros(shp))
    rmax, sweeps = [], []
    R.call("calvel")
    it = 0
    while True:  # press.for:441-472
        it += 1
        R.call("calmas")
        rmax.append(M.v_rmax)
        R.call("sipsol", 44)
        sweeps.append(M.v_nsweep)
        for ib in range(len(descs)):
            p = R.get_field("p", ib)
            pp = R.get_field("pp", ib)
            R.put_field("p", ib, p + (pp - 0.0))
            R.put_field("pp", ib, np.zeros_like(pp))
        R.call("exchange", 4)
        R.call("pbound")
        R.call("calvel")
        if not it < SIP_NITER:
            break
    out["rmax"] = np.array(rmax)
    out["nsweep"] = np.array(sweeps)
    for ib in range(len(descs)):
        for k in ("p", "u", "v", "w"):
            out["%s_out_%d" % (k, ib)] = R.get_field(k, ib)
        if not np.isfinite(out["p_out_%d" % ib]).all():
            raise RuntimeError("%s: the reference produced non-finite values" % name)
    return out


def main(prefix=""):
    """Write every fixture whose name starts with prefix (all by default)."""
    for name in CASES:
        if not name.startswith(prefix):
            continue
        data = run_case(name)
        np.savez_compressed(os.path.join(HERE, "mgkcyc_%s.npz" % name), **data)
        print("wrote", name)
    for name in PROJ_CASES:
        if not ("project_" + name).startswith(prefix):
            continue
        data = run_projection_case(name)
        np.savez_compressed(os.path.join(HERE, "project_%s.npz" % name), **data)
        print("wrote project", name)
    for name in SIP_CASES:
        if not ("sip_" + name).startswith(prefix):
            continue
        data = run_sip_case(name)
        np.savez_compressed(os.path.join(HERE, "sip_%s.npz" % name), **data)
        print("wrote sip", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "")
