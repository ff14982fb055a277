"""The mixed solver's FP32 sweep options: over-relaxation (omega) and the
red-black order across block faces (rb_order = 1).

  * Two FP32 sweeps of every smoother variant with omega = 1.25 and
    rb_order = 1 are red-black SOR in one colour order over the union of the
    blocks (numpy in FP64: red cells of every block, then black cells of every
    block, each cell x + omega (gs - x)), within the FP32 tolerance, with walls
    and with periodic partners (across blocks, and a block its own partner).
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

W, P = 4, 5  # wall, periodic
FP32_RTOL = 2e-5
H = 1.0 / 32


def _global_rb_sor(u, f, om, sweeps, periodic=(False, False, False)):
    """Red-black SOR of the cell-centred 7-point operator over a whole (z, y, x)
    domain, red = x+y+z odd (1-based): walls have a zero face coefficient, a
    periodic axis (x, y, z order) wraps around."""
    a = 1.0 / (H * H)
    shape = u.shape
    cw = np.full(shape, a); ce = np.full(shape, a)
    cs = np.full(shape, a); cn = np.full(shape, a)
    cb = np.full(shape, a); ct = np.full(shape, a)
    if not periodic[0]:
        cw[:, :, 0] = 0; ce[:, :, -1] = 0
    if not periodic[1]:
        cs[:, 0, :] = 0; cn[:, -1, :] = 0
    if not periodic[2]:
        cb[0] = 0; ct[-1] = 0
    ap = -(cw + ce + cs + cn + cb + ct)
    z, y, x = np.indices(shape) + 1
    red = (x + y + z) % 2 == 1
    for _ in range(sweeps):
        for colour in (red, ~red):
            s = (cw * np.roll(u, 1, 2) + ce * np.roll(u, -1, 2) + cs * np.roll(u, 1, 1) +
                 cn * np.roll(u, -1, 1) + cb * np.roll(u, 1, 0) + ct * np.roll(u, -1, 0))
            u = np.where(colour, u + om * ((f - s) / ap - u), u)
    return u


def _part(a, d):
    ox, oy, oz = d.origin
    nx, ny, nz = d.n
    return a[oz:oz + nz, oy:oy + ny, ox:ox + nx]


def test_sweeps_are_global_red_black_sor(h3d):
    rng = np.random.default_rng(5)
    for nblk, n, bc in (((2, 2, 1), (32, 16, 16), [W] * 6), ((2, 1, 2), (64, 12, 8), [W] * 6),
                        ((2, 1, 1), (32, 16, 8), [P, P, W, W, W, W]),      # periodic partners across blocks
                        ((1, 2, 1), (16, 16, 8), [W, W, P, P, P, P])):     # a block its own partner in z
        periodic = (bc[0] == P, bc[2] == P, bc[4] == P)
        blocks = h3d.topology.block_grid(nblk, n, bc, [H] * 3, 2)
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
                # every block with its ghost layer cut from the wrapped union: ghosts
                # across block faces and periodic faces hold the cells they show
                # (wall ghosts have a zero coefficient)
                uw = np.pad(u, 1, mode="wrap")
                for ib, d in enumerate(blocks):
                    ox, oy, oz = d.origin
                    s.put_level(1, "phi", ib, uw[oz:oz + d.n[2] + 2, oy:oy + d.n[1] + 2, ox:ox + d.n[0] + 2])
                    s.put_level(1, "rhs", ib, _part(f, d))
                s.mgrelax(1, 2)
                ref = _global_rb_sor(u, f, 1.25, 2, periodic)
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
