"""ctypes wrapper of the CPU oracle (oracle/liboracle_h3d.so).

TEST INFRASTRUCTURE ONLY.  The oracle is a C restatement of the reference
multigrid path (src_v70/mgsolver.for, exchangepp.for, newsolv_mg.for,
alloc_dom.for:read_infodom); it checks the CUDA product path.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import it.

Arrays exchanged with the oracle use the canonical per-block layout shared
with the product library: a level-g iterate is float64 of shape
(nz+2, ny+2, nx+2) (x fastest, one ghost layer), a right-hand side is
(nz, ny, nx).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_h3d.so")


class BlockDesc(C.Structure):
    """Byte-identical to or_block_desc / h3d_block_desc."""

    _fields_ = [
        ("n", C.c_int32 * 3),
        ("ttc", C.c_int32 * 3),
        ("pl", C.c_int32),
        ("ngrid", C.c_int32),
        ("h", C.c_double * 3),
        ("nb_face", C.c_int32 * 6),
        ("nb_corner", C.c_int32 * 8),
        ("nb_edge", C.c_int32 * 12),
        ("nb_periodic", C.c_int32 * 6),
        ("bc", C.c_int32 * 6),
        ("rdiv", C.c_int32),
        ("origin", C.c_int32 * 3),
    ]


_lib = None


def build():
    """Compile the oracle with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, i32, dbl = C.c_void_p, C.c_int, C.c_double
        pd = C.POINTER(C.c_double)
        ppd = C.POINTER(pd)
        L.or_create.restype = vp
        L.or_create.argtypes = [i32, C.POINTER(BlockDesc), i32, i32, i32, i32, i32]
        L.or_destroy.argtypes = [vp]
        L.or_error.argtypes = [vp]
        L.or_error.restype = i32
        L.or_set_density.argtypes = [vp, i32, pd]
        L.or_coeff.argtypes = [vp]
        for nm in ("or_put_phi", "or_get_phi", "or_put_rhs", "or_get_rhs"):
            getattr(L, nm).argtypes = [vp, i32, i32, pd]
        L.or_get_coef.argtypes = [vp, i32, i32, i32, pd]
        L.or_mgrelax.argtypes = [vp, i32, i32]
        for nm in ("or_mgrestr", "or_mgcorr", "or_mgbound", "or_exchangepp", "or_exchbc_mgpp"):
            getattr(L, nm).argtypes = [vp, i32]
        L.or_vcycle.argtypes = [vp]
        L.or_scale_level_coef.argtypes = [vp, i32, dbl]
        L.or_set_coef.argtypes = [vp, i32, i32, i32, pd]
        L.or_mgkcyc.argtypes = [vp, ppd, ppd]
        L.or_residual.argtypes = [vp, ppd, ppd, ppd, pd, pd]
        L.or_residual.restype = dbl
        L.or_solve.argtypes = [vp, ppd, ppd, dbl, i32, i32, C.POINTER(C.c_int), pd, pd]
        L.or_solve.restype = i32
        L.or_calvel.argtypes = [vp, ppd, ppd, ppd, ppd, ppd, ppd, ppd, ppd, dbl, dbl]
        L.or_vel_exchange.argtypes = [vp, ppd]
        L.or_calmas.argtypes = [vp, ppd, ppd, ppd, dbl, ppd, pd]
        L.or_calmas.restype = dbl
        L.or_project.argtypes = [vp, ppd, ppd, ppd, ppd, ppd, ppd, ppd, ppd, dbl, dbl, dbl, i32, i32,
                                 C.POINTER(C.c_int), pd, pd, pd]
        L.or_project.restype = i32
        L.or_sipsol.argtypes = [vp, ppd, ppd, i32, pd]
        L.or_sipsol.restype = i32
        L.or_pressure_1sweep.argtypes = [vp, ppd, ppd, ppd, ppd, ppd, ppd, ppd, dbl, dbl, dbl, i32, i32,
                                         C.POINTER(C.c_int), C.POINTER(C.c_int), pd]
        L.or_pressure_1sweep.restype = i32
        L.or_topology.argtypes = [i32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(BlockDesc)]
        L.or_topology.restype = i32
        L.or_set_threads.argtypes = [i32]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ptrs(arrs):
    P = C.POINTER(C.c_double)
    return (P * len(arrs))(*[_dp(a) for a in arrs])


def topology(ext, bc, h, ngrid):
    """read_infodom restatement: ext is (nblocks, 6) int (xs, xe, ys, ye, zs, ze)."""
    ext = np.ascontiguousarray(ext, dtype=np.int32)
    nb = ext.shape[0]
    bcv = np.ascontiguousarray(bc, dtype=np.int32)
    out = (BlockDesc * nb)()
    rc = lib().or_topology(nb, ext.ctypes.data_as(C.POINTER(C.c_int32)),
                           bcv.ctypes.data_as(C.POINTER(C.c_int32)), out)
    if rc != 0:
        raise ValueError("ambiguous block topology")
    for d in out:
        d.ngrid = ngrid
        d.rdiv = 1
        d.pl = 1
        for a in range(3):
            d.h[a] = float(h[a])
            d.ttc[a] = d.n[a] + 2
    return out


class Oracle:
    """The reference multigrid as a CPU object (one instance per problem)."""

    def __init__(self, descs, ngrd, mg_itrsch=3, irestr=2, iproln=1, lsm=False, threads=1):
        self.descs = descs
        self.nb = len(descs)
        self.ngrd = ngrd
        arr = (BlockDesc * self.nb)(*descs)
        self._h = lib().or_create(self.nb, arr, ngrd, mg_itrsch, irestr, iproln, int(bool(lsm)))
        if lib().or_error(self._h):
            lib().or_destroy(self._h)
            self._h = None
            raise ValueError("configuration rejected by the oracle")
        lib().or_set_threads(threads)

    def close(self):
        if self._h:
            lib().or_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # shapes --------------------------------------------------------------
    def dims(self, g, ib):
        n = self.descs[ib].n
        s = 2 ** (min(g, self.descs[ib].ngrid) - 1)  # level clamp, mgsolver.for:392-400
        return (n[2] // s, n[1] // s, n[0] // s)

    # reference routines -------------------------------------------------
    def set_density(self, ib, dens):
        d = np.ascontiguousarray(dens, dtype=np.float64)
        lib().or_set_density(self._h, ib, _dp(d))

    def coeff(self):
        lib().or_coeff(self._h)

    def put_phi(self, g, ib, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        lib().or_put_phi(self._h, g, ib, _dp(a))

    def get_phi(self, g, ib):
        nz, ny, nx = self.dims(g, ib)
        a = np.empty((nz + 2, ny + 2, nx + 2))
        lib().or_get_phi(self._h, g, ib, _dp(a))
        return a

    def put_rhs(self, g, ib, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        lib().or_put_rhs(self._h, g, ib, _dp(a))

    def get_rhs(self, g, ib):
        a = np.empty(self.dims(g, ib))
        lib().or_get_rhs(self._h, g, ib, _dp(a))
        return a

    def get_coef(self, g, ib, s):
        a = np.empty(self.dims(g, ib))
        lib().or_get_coef(self._h, g, ib, s, _dp(a))
        return a

    def set_coef(self, g, ib, s, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        lib().or_set_coef(self._h, g, ib, s, _dp(a))

    def scale_level_coef(self, g, s):
        lib().or_scale_level_coef(self._h, g, s)

    def mgrelax(self, g, it):
        lib().or_mgrelax(self._h, g, it)

    def mgrestr(self, g):
        lib().or_mgrestr(self._h, g)

    def mgcorr(self, g):
        lib().or_mgcorr(self._h, g)

    def mgbound(self, g):
        lib().or_mgbound(self._h, g)

    def exchangepp(self, g):
        lib().or_exchangepp(self._h, g)

    def vcycle(self):
        lib().or_vcycle(self._h)

    def mgkcyc(self, pp, su):
        pp = [np.ascontiguousarray(a, dtype=np.float64) for a in pp]
        su = [np.ascontiguousarray(a, dtype=np.float64) for a in su]
        lib().or_mgkcyc(self._h, _ptrs(pp), _ptrs(su))
        return pp

    def residual(self, p, b):
        p = [np.ascontiguousarray(a, dtype=np.float64).copy() for a in p]
        b = [np.ascontiguousarray(a, dtype=np.float64) for a in b]
        r = [np.empty_like(a) for a in b]
        bb = C.c_double()
        rinf = C.c_double()
        rr = lib().or_residual(self._h, _ptrs(p), _ptrs(b), _ptrs(r), C.byref(bb), C.byref(rinf))
        return r, rr, bb.value, rinf.value

    def solve(self, p, b, tol=1e-8, maxcy=200, stop_rule=0):
        p = [np.ascontiguousarray(a, dtype=np.float64).copy() for a in p]
        b = [np.ascontiguousarray(a, dtype=np.float64) for a in b]
        cyc = C.c_int()
        rel = C.c_double()
        hist = np.zeros(maxcy + 1)
        st = lib().or_solve(self._h, _ptrs(p), _ptrs(b), tol, maxcy, stop_rule,
                            C.byref(cyc), C.byref(rel), _dp(hist))
        return dict(p=p, status=st, cycles=cyc.value, relres=rel.value,
                    history=hist[: cyc.value + 1])

    # projection (press.for:2-144, newsolv_mg.for:2-93) ----------------------
    def _dens_ptrs(self, dens):
        if dens is None:
            return None, _ptrs([np.zeros(1)] * self.nb)
        d = [np.ascontiguousarray(a, dtype=np.float64) for a in dens]
        return d, _ptrs(d)

    def calvel(self, u, v, w, us, vs, ws, p, dt, alfapr=1.0, dens=None):
        """calvel followed by its exchange(1..3); u, v, w (canonical face
        arrays) are updated in place and returned."""
        u, v, w = ([np.ascontiguousarray(a, dtype=np.float64).copy() for a in f] for f in (u, v, w))
        us, vs, ws, p = ([np.ascontiguousarray(a, dtype=np.float64) for a in f] for f in (us, vs, ws, p))
        keep, dp = self._dens_ptrs(dens)
        lib().or_calvel(self._h, _ptrs(u), _ptrs(v), _ptrs(w), _ptrs(us), _ptrs(vs), _ptrs(ws), _ptrs(p), dp,
                        dt, alfapr)
        for f in (u, v, w):
            lib().or_vel_exchange(self._h, _ptrs(f))
        return u, v, w

    def calmas(self, u, v, w, dt):
        """(su per block (nz, ny, nx), sum su^2, rmax)."""
        u, v, w = ([np.ascontiguousarray(a, dtype=np.float64) for a in f] for f in (u, v, w))
        su = [np.empty(self.dims(1, ib)) for ib in range(self.nb)]
        rmax = C.c_double()
        ss = lib().or_calmas(self._h, _ptrs(u), _ptrs(v), _ptrs(w), dt, _ptrs(su), C.byref(rmax))
        return su, ss, rmax.value

    def project(self, p, u, v, w, us, vs, ws, dt, alfapr=1.0, dens=None, tol=1e-8, maxcy=200, stop_rule=0):
        p, u, v, w = ([np.ascontiguousarray(a, dtype=np.float64).copy() for a in f] for f in (p, u, v, w))
        us, vs, ws = ([np.ascontiguousarray(a, dtype=np.float64) for a in f] for f in (us, vs, ws))
        keep, dp = self._dens_ptrs(dens)
        cyc = C.c_int()
        rel = C.c_double()
        rmax = C.c_double()
        hist = np.zeros(maxcy + 1)
        st = lib().or_project(self._h, _ptrs(p), _ptrs(u), _ptrs(v), _ptrs(w), _ptrs(us), _ptrs(vs), _ptrs(ws), dp,
                              dt, alfapr, tol, maxcy, stop_rule, C.byref(cyc), C.byref(rel), C.byref(rmax),
                              _dp(hist))
        return dict(p=p, u=u, v=v, w=w, status=st, cycles=cyc.value, relres=rel.value, rmax=rmax.value,
                    history=hist[: cyc.value + 1])

    # SIP (sipsol.for:2-205, press.for:382-519) -----------------------------
    def sipsol(self, pp, su, nswp):
        """pp canonical (in/out copy returned), su interior: (pp, nsweep, sum|res| per sweep)."""
        pp = [np.ascontiguousarray(a, dtype=np.float64).copy() for a in pp]
        su = [np.ascontiguousarray(a, dtype=np.float64) for a in su]
        hist = np.zeros(nswp)
        ns = lib().or_sipsol(self._h, _ptrs(pp), _ptrs(su), nswp, _dp(hist))
        return pp, ns, hist[:ns]

    def pressure_1sweep(self, p, u, v, w, us, vs, ws, dt, alfapr=1.0, eps=1e-8, niter=10, nswp=50):
        p, u, v, w = ([np.ascontiguousarray(a, dtype=np.float64).copy() for a in f] for f in (p, u, v, w))
        us, vs, ws = ([np.ascontiguousarray(a, dtype=np.float64) for a in f] for f in (us, vs, ws))
        it, ns = C.c_int(), C.c_int()
        hist = np.zeros(niter)
        lib().or_pressure_1sweep(self._h, _ptrs(p), _ptrs(u), _ptrs(v), _ptrs(w), _ptrs(us), _ptrs(vs), _ptrs(ws),
                                 dt, alfapr, eps, niter, nswp, C.byref(it), C.byref(ns), _dp(hist))
        return dict(p=p, u=u, v=v, w=w, iters=it.value, nsweeps=ns.value, history=hist[:it.value])
