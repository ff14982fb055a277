"""Host-side mirror of the reference's multigrid pressure interface.

`MultigridSolver` keeps the subroutine names of Hydro3D v7.0's multigrid path
and their argument meaning:

    coeff()                        mgsolver.for:2-224
    mgkcyc(pp, su)                 mgsolver.for:226-372   (one V-cycle)
    newsolv_mg(p, b, ...)          newsolv_mg.for:2-93    (outer defect correction)
    project(p, u, v, w, ustar, vstar, wstar, dt, ...)
                                   newsolv_mg.for:2-93 with calvel/calmas (press.for:2-144)
    calvel(dt, alfapr) / calmas(dt) / pbound()
                                   press.for:2-207 on the resident fields
    sipsol(nswp) / pressure_1sweep(dt, ...)
                                   sipsol.for:2-205, press.for:382-519 (the SIP path)
    mgrelax(g, it) / mgrestr(g) / mgcorr(g) / mgbound(g) / exchangepp(g)
                                   mgsolver.for:374-997, exchangepp.for:2-2835

Host fields are numpy float64 arrays laid out like the Fortran `dom(ib)` arrays:
shape (ttc_k, ttc_j, ttc_i) in C order == Fortran (ttc_i, ttc_j, ttc_k), with
`pl` ghost layers.  Every call goes through the C ABI of libh3dmg.so; there is
no CPU code path.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import H3DError, check


def host_field(d) -> np.ndarray:
    """A zero host field for block descriptor d (Fortran dims ttc, pl ghosts)."""
    return np.zeros((d.ttc[2], d.ttc[1], d.ttc[0]))


def interior(a: np.ndarray, d) -> np.ndarray:
    p = d.pl
    return a[p:p + d.n[2], p:p + d.n[1], p:p + d.n[0]]


def with_ghost(a: np.ndarray, d) -> np.ndarray:
    """The interior plus the first ghost layer (what the MG path reads/writes)."""
    p = d.pl
    return a[p - 1:p + d.n[2] + 1, p - 1:p + d.n[1] + 1, p - 1:p + d.n[0] + 1]


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ptrs(arrs):
    P = C.POINTER(C.c_double)
    return (P * len(arrs))(*[_dp(a) for a in arrs])


class MultigridSolver:
    """One multi-block pressure-Poisson problem resident on one GPU."""

    def __init__(self, blocks: Sequence, ngrd_gl: int, mg_itrsch: int = 3, irestr: int = 2, iproln: int = 1,
                 maxcy: int = 30, precision: str = "fp64", var_coef: bool = False, device: int = 0,
                 coarse_sweeps: int = 0, inner_cycles: int = 0, use_graph: bool = True, coarse_op: int = 0,
                 coarse_direct: bool = False, rb_order: int = 0, omega: float = 0.0):
        self.L = _lib.lib()
        self.blocks = list(blocks)
        self._arr = (_lib.BlockDesc * len(self.blocks))(*self.blocks)
        desc = _lib.MGDesc()
        desc.nblocks = len(self.blocks)
        desc.ngrd_gl = ngrd_gl
        desc.mg_itrsch = mg_itrsch
        desc.irestr = irestr
        desc.iproln = iproln
        desc.maxcy = maxcy
        desc.precision = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}[precision]
        desc.var_coef = int(bool(var_coef))
        desc.device = device
        desc.coarse_sweeps = coarse_sweeps
        desc.inner_cycles = inner_cycles
        desc.use_graph = int(bool(use_graph))
        desc.coarse_op = coarse_op
        desc.coarse_direct = int(bool(coarse_direct))
        desc.rb_order = int(rb_order)
        desc.omega = float(omega)
        desc.blocks = self._arr
        self.ngrd = ngrd_gl
        self.precision = precision
        self.maxcy = maxcy
        self._h = C.c_void_p()
        rc = self.L.h3d_mg_create(C.byref(self._h), C.byref(desc))
        if rc != _lib.H3D_OK:
            msg = self.L.h3d_mg_last_error(None).decode()
            raise H3DError(rc, f"h3d_mg_create: {self.L.h3d_mg_strerror(rc).decode()}: {msg}")

    # life cycle ----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self.L.h3d_mg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        return check(rc, self._h, what)

    # set-up --------------------------------------------------------------
    def set_density(self, ib: int, dens: np.ndarray):
        dens = np.ascontiguousarray(dens, dtype=np.float64)
        self._check(self.L.h3d_mg_set_density(self._h, ib, _dp(dens)), "h3d_mg_set_density")

    def coeff(self):
        self._check(self.L.h3d_mg_coeff(self._h), "h3d_mg_coeff")

    # drop-in calls -------------------------------------------------------
    def mgkcyc(self, pp: List[np.ndarray], su: List[np.ndarray]):
        """One V-cycle: pp (host fields, in/out), su (host fields)."""
        for a in list(pp) + list(su):
            assert a.dtype == np.float64 and a.flags.c_contiguous
        self._check(self.L.h3d_mg_mgkcyc(self._h, _ptrs(pp), _ptrs(su)), "h3d_mg_mgkcyc")

    @staticmethod
    def _opts(tol, maxcy, stop_rule, remove_mean, history):
        o = _lib.SolveOpts()
        o.tol = tol
        o.maxcy = maxcy
        o.stop_rule = stop_rule
        o.remove_mean = int(bool(remove_mean))
        o.record_history = int(bool(history))
        return o

    def _info(self, rc, info, history, raise_diverged=True):
        out = {k: getattr(info, k) for k, _ in _lib.SolveInfo._fields_}
        out["converged"] = rc == _lib.H3D_OK
        out["status"] = rc
        if history:
            n = C.c_int32()
            self.L.h3d_mg_history(self._h, None, 0, C.byref(n))
            buf = np.zeros(n.value)
            self.L.h3d_mg_history(self._h, _dp(buf), n.value, C.byref(n))
            out["history"] = buf
        if rc not in (_lib.H3D_OK, _lib.H3D_ERR_NOT_CONVERGED) and (raise_diverged or rc != _lib.H3D_ERR_DIVERGED):
            self._check(rc, "solve")
        return out

    def newsolv_mg(self, p: List[np.ndarray], b: List[np.ndarray], tol: float = 1e-8, maxcy: int = 0,
                   stop_rule: int = 0, remove_mean: bool = False, history: bool = False) -> dict:
        """Solve A p = b (host fields, p in/out) by FP64 defect correction.

        Like the reference, an exhausted cycle budget is reported (converged
        False), not raised; a diverged solve raises."""
        opts = self._opts(tol, maxcy, stop_rule, remove_mean, history)
        info = _lib.SolveInfo()
        rc = self.L.h3d_mg_newsolv(self._h, _ptrs(p), _ptrs(b), C.byref(opts), C.byref(info))
        return self._info(rc, info, history)

    def project(self, p: List[np.ndarray], u: List[np.ndarray], v: List[np.ndarray], w: List[np.ndarray],
                ustar: List[np.ndarray], vstar: List[np.ndarray], wstar: List[np.ndarray], dt: float,
                alfapr: float = 1.0, tol: float = 1e-8, maxcy: int = 0, stop_rule: int = 0,
                history: bool = False) -> dict:
        """newsolv_mg with the velocities: p, u, v, w host fields in/out,
        ustar, vstar, wstar host fields in.  stop_rule 1 is the reference's
        rmax < tol (after at least two cycles); 0 is ||su|| <= tol ||su_0||."""
        for a in list(p) + list(u) + list(v) + list(w) + list(ustar) + list(vstar) + list(wstar):
            assert a.dtype == np.float64 and a.flags.c_contiguous
        opts = self._opts(tol, maxcy, stop_rule, False, history)
        info = _lib.SolveInfo()
        rc = self.L.h3d_mg_project(self._h, _ptrs(p), _ptrs(u), _ptrs(v), _ptrs(w), _ptrs(ustar), _ptrs(vstar),
                                   _ptrs(wstar), dt, alfapr, C.byref(opts), C.byref(info))
        return self._info(rc, info, history)

    def project_resident(self, dt: float, alfapr: float = 1.0, tol: float = 1e-8, maxcy: int = 0,
                         stop_rule: int = 0, history: bool = False) -> dict:
        opts = self._opts(tol, maxcy, stop_rule, False, history)
        info = _lib.SolveInfo()
        rc = self.L.h3d_mg_project_resident(self._h, dt, alfapr, C.byref(opts), C.byref(info))
        return self._info(rc, info, history)

    def sipsol(self, nswp: int):
        """sipsol(44) on the resident 'pp' with rhs 'b': (nsweep, last sum |res|)."""
        ns, ra = C.c_int32(), C.c_double()
        self._check(self.L.h3d_mg_sipsol(self._h, nswp, C.byref(ns), C.byref(ra)), "h3d_mg_sipsol")
        return ns.value, ra.value

    def pressure_1sweep(self, dt: float, alfapr: float = 1.0, eps: float = 1e-8, niter: int = 10,
                        nswp: int = 50) -> dict:
        """The SIP pressure loop (press.for:382-519) on the resident fields;
        history = rmax of every calmas."""
        info = _lib.SolveInfo()
        rc = self.L.h3d_mg_pressure_1sweep(self._h, dt, alfapr, eps, niter, nswp, C.byref(info))
        return self._info(rc, info, True)

    def calvel(self, dt: float, alfapr: float = 1.0):
        self._check(self.L.h3d_mg_calvel(self._h, dt, alfapr), "h3d_mg_calvel")

    def calmas(self, dt: float):
        """(rmax, sum su^2); su lands in the resident field 'b'."""
        rmax, s2 = C.c_double(), C.c_double()
        self._check(self.L.h3d_mg_calmas(self._h, dt, C.byref(rmax), C.byref(s2)), "h3d_mg_calmas")
        return rmax.value, s2.value

    def pbound(self):
        self._check(self.L.h3d_mg_pbound(self._h), "h3d_mg_pbound")

    # resident operation --------------------------------------------------
    FIELDS = {"p": _lib.FIELD_P, "b": _lib.FIELD_B, "u": _lib.FIELD_U, "v": _lib.FIELD_V, "w": _lib.FIELD_W,
              "ustar": _lib.FIELD_USTAR, "vstar": _lib.FIELD_VSTAR, "wstar": _lib.FIELD_WSTAR, "pp": _lib.FIELD_PP}

    def upload(self, field: str, ib: int, host: np.ndarray):
        f = self.FIELDS[field]
        host = np.ascontiguousarray(host, dtype=np.float64)
        self._check(self.L.h3d_mg_upload(self._h, f, ib, _dp(host)), "h3d_mg_upload")

    def download(self, field: str, ib: int, host: np.ndarray):
        f = self.FIELDS[field]
        assert host.dtype == np.float64 and host.flags.c_contiguous
        self._check(self.L.h3d_mg_download(self._h, f, ib, _dp(host)), "h3d_mg_download")

    def zero_field(self, field: str):
        f = {"p": _lib.FIELD_P, "b": _lib.FIELD_B}[field]
        self._check(self.L.h3d_mg_zero_field(self._h, f), "h3d_mg_zero_field")

    def solve_resident(self, tol: float = 1e-8, maxcy: int = 0, stop_rule: int = 0, remove_mean: bool = False,
                       history: bool = False, raise_diverged: bool = True) -> dict:
        """Solve with p and b resident.  A diverged solve raises unless
        raise_diverged is False (then info["status"] is H3D_ERR_DIVERGED)."""
        opts = self._opts(tol, maxcy, stop_rule, remove_mean, history)
        info = _lib.SolveInfo()
        rc = self.L.h3d_mg_solve_resident(self._h, C.byref(opts), C.byref(info))
        return self._info(rc, info, history, raise_diverged)

    def residual(self):
        rr, bb, ri = C.c_double(), C.c_double(), C.c_double()
        self._check(self.L.h3d_mg_residual(self._h, C.byref(rr), C.byref(bb), C.byref(ri)), "h3d_mg_residual")
        return rr.value, bb.value, ri.value

    def set_wait_limit(self, clocks: int):
        """Limit of the bounded device waits on this GPU (<= 0: the default)."""
        self._check(self.L.h3d_mg_set_wait_limit(self._h, int(clocks)), "h3d_mg_set_wait_limit")

    def wait_probe(self) -> int:
        """One bounded device wait that cannot complete: the status code
        (H3D_ERR_TIMEOUT once the limit has run out)."""
        return self.L.h3d_mg_wait_probe(self._h)

    def set_profiling(self, on: bool):
        self._check(self.L.h3d_mg_set_profiling(self._h, int(bool(on))), "h3d_mg_set_profiling")

    def smoother_bytes(self) -> float:
        v = C.c_double()
        self._check(self.L.h3d_mg_smoother_bytes(self._h, C.byref(v)), "h3d_mg_smoother_bytes")
        return v.value

    def set_smoother(self, g: int, variant: int, zchunk: int) -> bool:
        """Force smoother variant / z-chunk of level g; False if it cannot run there."""
        rc = self.L.h3d_mg_set_smoother(self._h, g, variant, zchunk)
        if rc == _lib.H3D_ERR_ARG:
            return False
        self._check(rc, "h3d_mg_set_smoother")
        return True

    def set_restriction(self, g: int, variant: int, zchunk: int) -> bool:
        """Force the restriction variant / coarse z-chunk into level g; False if it cannot run there."""
        rc = self.L.h3d_mg_set_restriction(self._h, g, variant, zchunk)
        if rc == _lib.H3D_ERR_ARG:
            return False
        self._check(rc, "h3d_mg_set_restriction")
        return True

    def get_restriction(self, g: int):
        v, z, n = C.c_int32(), C.c_int32(), C.c_int32()
        self._check(self.L.h3d_mg_get_restriction(self._h, g, C.byref(v), C.byref(z), C.byref(n)),
                    "h3d_mg_get_restriction")
        return v.value, z.value, n.value

    def get_smoother(self, g: int):
        v, z, n = C.c_int32(), C.c_int32(), C.c_int32()
        self._check(self.L.h3d_mg_get_smoother(self._h, g, C.byref(v), C.byref(z), C.byref(n)), "h3d_mg_get_smoother")
        return v.value, z.value, n.value

    # reference subroutines on the level state ----------------------------
    def level_dims(self, g: int, ib: int):
        d = self.blocks[ib]
        s = 2 ** (g - 1)
        return d.n[2] // s, d.n[1] // s, d.n[0] // s

    def put_level(self, g: int, field: str, ib: int, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        f = {"phi": 0, "rhs": 1}[field]
        self._check(self.L.h3d_mg_put_level(self._h, g, f, ib, _dp(a)), "h3d_mg_put_level")

    def get_level(self, g: int, field: str, ib: int) -> np.ndarray:
        nz, ny, nx = self.level_dims(g, ib)
        f = {"phi": 0, "rhs": 1}[field]
        a = np.empty((nz + 2, ny + 2, nx + 2)) if f == 0 else np.empty((nz, ny, nx))
        self._check(self.L.h3d_mg_get_level(self._h, g, f, ib, _dp(a)), "h3d_mg_get_level")
        return a

    def mgrelax(self, g: int, it: int):
        self._check(self.L.h3d_mg_mgrelax(self._h, g, it), "h3d_mg_mgrelax")

    def mgrestr(self, g: int):
        self._check(self.L.h3d_mg_mgrestr(self._h, g), "h3d_mg_mgrestr")

    def mgcorr(self, g: int):
        self._check(self.L.h3d_mg_mgcorr(self._h, g), "h3d_mg_mgcorr")

    def mgbound(self, g: int):
        self._check(self.L.h3d_mg_mgbound(self._h, g), "h3d_mg_mgbound")

    def exchangepp(self, g: int):
        self._check(self.L.h3d_mg_exchangepp(self._h, g), "h3d_mg_exchangepp")

    def vcycle(self):
        self._check(self.L.h3d_mg_vcycle(self._h), "h3d_mg_vcycle")


def halo_expr(blocks: Sequence, g: int, kind: int):
    """Expression form of level g's fill (host-only; see h3d_halo_expr):
    returns nodes (n, 9) uint32, dst, src."""
    L = _lib.lib()
    arr = (_lib.BlockDesc * len(blocks))(*blocks)
    n = C.c_int64()
    nn = C.c_int64()
    check(L.h3d_halo_expr(len(blocks), arr, g, kind, None, 0, C.byref(nn), None, None, 0, C.byref(n)), None,
          "h3d_halo_expr")
    nodes = np.zeros((nn.value, 9), dtype=np.uint32)
    dst = np.zeros(n.value, dtype=np.uint32)
    src = np.zeros(n.value, dtype=np.uint32)
    pu = C.POINTER(C.c_uint32)
    check(L.h3d_halo_expr(len(blocks), arr, g, kind, nodes.ctypes.data_as(pu), nn.value, C.byref(nn),
                          dst.ctypes.data_as(pu), src.ctypes.data_as(pu), n.value, C.byref(n)), None, "h3d_halo_expr")
    return nodes, dst, src


def halo_table(blocks: Sequence, g: int, kind: int):
    """Ghost gather table of level g (host-only; see h3d_halo_table)."""
    L = _lib.lib()
    arr = (_lib.BlockDesc * len(blocks))(*blocks)
    n = C.c_int64()
    check(L.h3d_halo_table(len(blocks), arr, g, kind, None, None, 0, C.byref(n)), None, "h3d_halo_table")
    dst = np.zeros(n.value, dtype=np.uint32)
    src = np.zeros(n.value, dtype=np.uint32)
    check(L.h3d_halo_table(len(blocks), arr, g, kind, dst.ctypes.data_as(C.POINTER(C.c_uint32)),
                           src.ctypes.data_as(C.POINTER(C.c_uint32)), n.value, C.byref(n)), None, "h3d_halo_table")
    return dst, src
