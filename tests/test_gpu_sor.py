"""The mixed solver's FP32 sweep options: over-relaxation (omega) and the
red-black order across block faces (rb_order = 1).

  * Two FP32 sweeps of every smoother variant with omega = 1.25 and
    rb_order = 1 are red-black SOR in one colour order over the union of the
    blocks (numpy in FP64: red cells of every block, then black cells of every
    block, each cell x + omega (gs - x)), within the FP32 tolerance, with walls
    and with periodic partners (across blocks, and a block its own partner),
    and with L_LSM face coefficients from a density field.
  * With those options the configuration-3 layout (4 x 2 x 2 blocks, here of
    32^3) meets 1e-8 in fewer V-cycles than with the reference's per-block
    order and Gauss-Seidel, and its solution is as close to the converged FP64
    one; two variable-density blocks meet it in no more cycles.
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


def _mirrored_density():
    """1 to 10, mirrored about x = 1/2 (the face of two 32^3 blocks side by
    side): the reference's coefficient of a block-face face takes the density
    of the block's own cell (mgsolver.for:78-184), so the two sides agree, and
    the operator is the interior formula everywhere, only where the density
    does not jump across the face."""
    z, y, x = np.meshgrid(*[(np.arange(k) + 0.5) / k for k in (32, 32, 32)], indexing="ij")
    half = 1.0 + 9.0 * (0.5 + 0.5 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) * np.sin(np.pi * z))
    return np.concatenate([half, half[:, :, ::-1]], axis=2)


def _density_fields(h3d, blocks, rho):
    rho_g = np.pad(rho, 1, mode="edge")  # ghosts across the block face: the neighbour's cells
    out = []
    for d in blocks:
        a = h3d.host_field(d)
        ox, oy, oz = d.origin
        h3d.with_ghost(a, d)[...] = rho_g[oz:oz + d.n[2] + 2, oy:oy + d.n[1] + 2, ox:ox + d.n[0] + 2]
        out.append(a)
    return out


def test_variable_density_sweeps_are_global_red_black_sor(h3d):
    """Two FP32 sweeps with L_LSM coefficients (every variable-coefficient
    smoother variant) in the order across blocks with omega = 1.25: numpy
    red-black SOR with the face coefficients h / (mean of the two densities),
    zero at walls."""
    blocks = h3d.topology.block_grid((2, 1, 1), (32, 32, 32), [W] * 6, [H] * 3, 2)
    rho = _mirrored_density()
    s = h3d.MultigridSolver(blocks, 2, precision="mixed", var_coef=True, coarse_op=1, use_graph=False,
                            omega=1.25, rb_order=1)
    for ib, a in enumerate(_density_fields(h3d, blocks, rho)):
        s.set_density(ib, a)
    s.coeff()
    shape = rho.shape
    cw = np.zeros(shape); ce = np.zeros(shape); cs = np.zeros(shape)
    cn = np.zeros(shape); cb = np.zeros(shape); ct = np.zeros(shape)
    cw[:, :, 1:] = H / (0.5 * (rho[:, :, 1:] + rho[:, :, :-1])); ce[:, :, :-1] = cw[:, :, 1:]
    cs[:, 1:, :] = H / (0.5 * (rho[:, 1:, :] + rho[:, :-1, :])); cn[:, :-1, :] = cs[:, 1:, :]
    cb[1:] = H / (0.5 * (rho[1:] + rho[:-1])); ct[:-1] = cb[1:]
    ap = -(cw + ce + cs + cn + cb + ct)
    z, y, x = np.indices(shape) + 1
    red = (x + y + z) % 2 == 1
    rng = np.random.default_rng(13)
    _, _, nvar = s.get_smoother(1)
    tried = 0
    for v in range(nvar):
        for zc in (3, 16):
            if not s.set_smoother(1, v, zc):
                continue
            tried += 1
            u = rng.standard_normal(shape)
            f = rng.standard_normal(shape)
            uw = np.pad(u, 1, mode="wrap")
            for ib, d in enumerate(blocks):
                ox, oy, oz = d.origin
                s.put_level(1, "phi", ib, uw[oz:oz + d.n[2] + 2, oy:oy + d.n[1] + 2, ox:ox + d.n[0] + 2])
                s.put_level(1, "rhs", ib, _part(f, d))
            s.mgrelax(1, 2)
            ref = u.copy()
            for _ in range(2):
                for colour in (red, ~red):
                    nb = (cw * np.roll(ref, 1, 2) + ce * np.roll(ref, -1, 2) + cs * np.roll(ref, 1, 1) +
                          cn * np.roll(ref, -1, 1) + cb * np.roll(ref, 1, 0) + ct * np.roll(ref, -1, 0))
                    ref = np.where(colour, ref + 1.25 * ((f - nb) / ap - ref), ref)
            scale = np.abs(ref).max()
            for ib, d in enumerate(blocks):
                got = s.get_level(1, "phi", ib)[1:-1, 1:-1, 1:-1]
                np.testing.assert_allclose(got, _part(ref, d), rtol=FP32_RTOL, atol=FP32_RTOL * scale,
                                           err_msg="variant %d z-chunk %d block %d" % (v, zc, ib))
    assert tried >= 2
    s.close()


def test_variable_density_across_blocks(h3d):
    """Two blocks with L_LSM coefficients from a smooth density (1 to 10): the
    red cells next to the block face are computed ahead with the face
    coefficients (k_red_ahead<VAR>), and the mixed solve with omega = 1.25 in
    the order across blocks meets 1e-8 no later than Gauss-Seidel in the
    reference's order, within an order of magnitude of the error of an FP64
    solve stopped at the same tolerance (over-relaxed cycles leave a smoother
    residual: at equal ||r|| the error is larger; measured 3.5x here)."""
    blocks = h3d.topology.block_grid((2, 1, 1), (32, 32, 32), [W] * 6, [H] * 3, 4)
    rho = _mirrored_density()
    rng = np.random.default_rng(9)
    f = rng.standard_normal(rho.shape)
    f -= f.mean()
    dens = _density_fields(h3d, blocks, rho)
    b = []
    for d in blocks:
        c = h3d.host_field(d)
        h3d.interior(c, d)[...] = _part(f, d) * H ** 3  # L_LSM rhs carries the cell volume
        b.append(c)

    def solve(precision, tol, **kw):
        s = h3d.MultigridSolver(blocks, 4, precision=precision, var_coef=True, coarse_op=1, coarse_sweeps=32,
                                maxcy=400, **kw)
        for ib in range(len(blocks)):
            s.set_density(ib, dens[ib])
        s.coeff()
        p = [h3d.host_field(d) for d in blocks]
        info = s.newsolv_mg(p, b, tol=tol, maxcy=400)
        s.close()
        assert info["converged"], info
        return [h3d.interior(x, d) for x, d in zip(p, blocks)], info

    exact, _ = solve("fp64", 1e-11)
    plain, _ = solve("fp64", 1e-8)
    _, ib = solve("mixed", 1e-8)
    opt, io = solve("mixed", 1e-8, omega=1.25, rb_order=1)
    assert io["cycles"] <= ib["cycles"], (io["cycles"], ib["cycles"])
    ep = mean_removed_rel(plain, exact)
    eo = mean_removed_rel(opt, exact)
    assert eo <= max(10.0 * ep, 1e-8), (eo, ep)
