"""The mixed solver's FP32 sweep options: over-relaxation (omega) and the
red-black order across block faces (rb_order = 1).

  * Two FP32 sweeps of every smoother variant with omega = 1.25 and
    rb_order = 1 are red-black SOR in one colour order over the union of the
    blocks (numpy in FP64: red cells of every block, then black cells of every
    block, each cell x + omega (gs - x)), within the FP32 tolerance.
  * With those options the configuration-3 layout (4 x 2 x 2 blocks, here of
    32^3) meets 1e-8 in fewer V-cycles than with the reference's per-block
    order and Gauss-Seidel, and its solution is as close to the converged FP64
    one.
  * The descriptor rejects omega outside [0, 2) and rb_order outside {0, 1}
    (host check, no device work: see tests/test_abi.py).
"""
import numpy as np
import pytest

from tests.helpers import interior_of_host, mean_removed_rel

pytestmark = pytest.mark.gpu

W = 4
FP32_RTOL = 2e-5
H = 1.0 / 32


def _global_rb_sor(u, f, om, sweeps):
    """Red-black SOR of the cell-centred 7-point operator (walls: zero face
    coefficient) over a whole (z, y, x) domain, red = x+y+z odd (1-based)."""
    a = 1.0 / (H * H)
    shape = u.shape
    cw = np.full(shape, a); cw[:, :, 0] = 0
    ce = np.full(shape, a); ce[:, :, -1] = 0
    cs = np.full(shape, a); cs[:, 0, :] = 0
    cn = np.full(shape, a); cn[:, -1, :] = 0
    cb = np.full(shape, a); cb[0] = 0
    ct = np.full(shape, a); ct[-1] = 0
    ap = -(cw + ce + cs + cn + cb + ct)
    z, y, x = np.indices(shape) + 1
    red = (x + y + z) % 2 == 1
    for _ in range(sweeps):
        for colour in (red, ~red):
            g = np.pad(u, 1)
            s = (cw * g[1:-1, 1:-1, :-2] + ce * g[1:-1, 1:-1, 2:] + cs * g[1:-1, :-2, 1:-1] +
                 cn * g[1:-1, 2:, 1:-1] + cb * g[:-2, 1:-1, 1:-1] + ct * g[2:, 1:-1, 1:-1])
            u = np.where(colour, u + om * ((f - s) / ap - u), u)
    return u


def _part(a, d):
    ox, oy, oz = d.origin
    nx, ny, nz = d.n
    return a[oz:oz + nz, oy:oy + ny, ox:ox + nx]


def test_sweeps_are_global_red_black_sor(h3d):
    rng = np.random.default_rng(5)
    for nblk, n in (((2, 2, 1), (32, 16, 16)), ((2, 1, 2), (64, 12, 8))):
        blocks = h3d.topology.block_grid(nblk, n, [W] * 6, [H] * 3, 2)
        s = h3d.MultigridSolver(blocks, 2, precision="mixed", use_graph=False, omega=1.25, rb_order=1)
        s.coeff()
        shape = (nblk[2] * n[2], nblk[1] * n[1], nblk[0] * n[0])
        _, _, nvar = s.get_smoother(1)
        tried = 0
        for v in range(nvar):
            for zc in (3, 16):
                if not s.set_smoother(1, v, zc):
                    continue
                tried += 1
                u = rng.standard_normal(shape)
                f = rng.standard_normal(shape)
                for ib, d in enumerate(blocks):
                    p = np.zeros((d.n[2] + 2, d.n[1] + 2, d.n[0] + 2))
                    p[1:-1, 1:-1, 1:-1] = _part(u, d)
                    s.put_level(1, "phi", ib, p)
                    s.put_level(1, "rhs", ib, _part(f, d))
                s.exchangepp(1)  # ghosts across block faces hold the neighbours' cells
                s.mgrelax(1, 2)
                ref = _global_rb_sor(u, f, 1.25, 2)
                scale = np.abs(ref).max()
                for ib, d in enumerate(blocks):
                    got = s.get_level(1, "phi", ib)[1:-1, 1:-1, 1:-1]
                    np.testing.assert_allclose(got, _part(ref, d), rtol=FP32_RTOL, atol=FP32_RTOL * scale,
                                               err_msg="variant %d z-chunk %d block %d" % (v, zc, ib))
        assert tried >= 4
        s.close()


def test_options_cut_cycles_at_equal_error(h3d):
    from hydro3d_b200 import synth
    prob = synth.config3(n=32, ngrid=5)

    def solve(precision, tol, **kw):
        s = h3d.MultigridSolver(prob.blocks, prob.ngrid, precision=precision, maxcy=400, coarse_sweeps=32,
                                coarse_direct=True, **kw)
        s.coeff()
        p = [x.copy() for x in prob.p0]
        info = s.newsolv_mg(p, prob.b, tol=tol, maxcy=400)
        s.close()
        assert info["converged"], info
        return p, info

    exact, _ = solve("fp64", 1e-12)
    base, ib = solve("mixed", 1e-8, inner_cycles=4)
    opt, io = solve("mixed", 1e-8, inner_cycles=3, omega=1.25, rb_order=1)
    assert io["cycles"] < ib["cycles"], (io["cycles"], ib["cycles"])

    def inner(fields):
        return [interior_of_host(x, d) for x, d in zip(fields, prob.blocks)]

    eb = mean_removed_rel(inner(base), inner(exact))
    eo = mean_removed_rel(inner(opt), inner(exact))
    assert eo <= max(eb, 1e-8), (eo, eb)
