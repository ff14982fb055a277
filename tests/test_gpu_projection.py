"""GPU parity of the projection (press.for:2-207, newsolv_mg.for:2-93)
through the C ABI: calvel with its exchange(1..3), calmas, and the whole
newsolv_mg loop with the velocities, against the oracle's restatement.

FP64 is compared bit for bit: velocities on every cell of the canonical
block (the cells neither side writes keep the same inputs), su and rmax,
the cycle count and the rmax history of the reference stop rule, and the
pressure on the interior and the face ghosts of the interior rows (the edge
and corner ghosts are not part of the projection's output: the device keeps
p + pp there, the oracle's level-1 exchange rewrites them).  The
mixed-precision projection is checked against the FP64 oracle's solution.
"""
import numpy as np
import pytest

from tests.helpers import mean_removed_rel, projection_fields, to_host, to_oracle_descs

pytestmark = pytest.mark.gpu

W, P = 4, 5
LAYOUTS = [
    ((1, 1, 1), (16, 16, 16), [W] * 6, 3),
    ((2, 2, 2), (8, 16, 8), [P, P, W, W, W, W], 3),
    ((3, 2, 2), (16, 8, 8), [W, W, P, P, W, W], 2),
    ((2, 1, 3), (8, 8, 16), [P] * 6, 3),
    ((1, 2, 1), (16, 8, 16), [W, W, W, W, P, P], 3),
]


def _pair(O, h3d, layout, lsm=False, precision="fp64", seed=11, dens_hi=1000.0, **kw):
    nblk, n, bc, ngrid = layout
    blocks = h3d.topology.block_grid(nblk, n, bc, [1.0 / 32] * 3, ngrid)
    s = h3d.MultigridSolver(blocks, ngrid, precision=precision, var_coef=lsm, **kw)
    orc = O.Oracle(to_oracle_descs(O, blocks), ngrid, 3, 2, 1, lsm=lsm)
    f = projection_fields(blocks, seed, lsm, dens_hi)
    if lsm:
        for ib, (d, x) in enumerate(zip(blocks, to_host(blocks, f["dens"]))):
            s.set_density(ib, x)
            orc.set_density(ib, f["dens"][ib][1:-1, 1:-1, 1:-1])
    s.coeff()
    orc.coeff()
    return blocks, s, orc, f


def _canon(h3d, host, d):
    return np.ascontiguousarray(h3d.with_ghost(host, d))


def _face_mask(a):
    """Interior cells and face ghosts (at most one ghost coordinate)."""
    nz, ny, nx = a.shape
    gz = (np.arange(nz) == 0) | (np.arange(nz) == nz - 1)
    gy = (np.arange(ny) == 0) | (np.arange(ny) == ny - 1)
    gx = (np.arange(nx) == 0) | (np.arange(nx) == nx - 1)
    cnt = gz[:, None, None].astype(int) + gy[None, :, None] + gx[None, None, :]
    return cnt <= 1


def _upload_all(s, blocks, f):
    for k, name in (("p", "p"), ("u", "u"), ("v", "v"), ("w", "w"), ("us", "ustar"), ("vs", "vstar"), ("ws", "wstar")):
        for ib, x in enumerate(to_host(blocks, f[k])):
            s.upload(name, ib, x)


@pytest.mark.parametrize("lsm", [False, True])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_calvel_bitexact(oracle_mod, h3d, layout, lsm):
    blocks, s, orc, f = _pair(oracle_mod, h3d, layout, lsm)
    _upload_all(s, blocks, f)
    dt, alfapr = 0.37, 0.9
    s.calvel(dt, alfapr)
    want = orc.calvel(f["u"], f["v"], f["w"], f["us"], f["vs"], f["ws"], f["p"], dt, alfapr,
                      dens=f["dens"] if lsm else None)
    for c, name in enumerate(("u", "v", "w")):
        for ib, d in enumerate(blocks):
            host = h3d.host_field(d)
            s.download(name, ib, host)
            got = _canon(h3d, host, d)
            assert np.array_equal(got, want[c][ib]), (name, ib, float(np.abs(got - want[c][ib]).max()))
    s.close()


@pytest.mark.parametrize("lsm", [False, True])
@pytest.mark.parametrize("layout", LAYOUTS[:3])
def test_calmas_bitexact(oracle_mod, h3d, layout, lsm):
    blocks, s, orc, f = _pair(oracle_mod, h3d, layout, lsm)
    _upload_all(s, blocks, f)
    dt = 0.37
    rmax, s2 = s.calmas(dt)
    su, ss, rmax_o = orc.calmas(f["u"], f["v"], f["w"], dt)
    assert rmax == rmax_o
    assert np.isclose(s2, ss, rtol=1e-12, atol=0)
    for ib, d in enumerate(blocks):
        host = h3d.host_field(d)
        s.download("b", ib, host)
        assert np.array_equal(h3d.interior(host, d), su[ib])
    s.close()


@pytest.mark.parametrize("lsm", [False, True])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_projection_fp64_bitexact(oracle_mod, h3d, layout, lsm):
    """The reference stop rule: the same cycles, the same rmax after every
    cycle, the same p, u, v, w.  The L_LSM density varies cell by cell in
    [1, 4]: with the reference's coarse levels (coefficients from the
    averaged density) a cell-by-cell 1000:1 field makes the loop diverge,
    the oracle's and the device's alike."""
    blocks, s, orc, f = _pair(oracle_mod, h3d, layout, lsm, dens_hi=4.0)
    dt, alfapr, eps = 0.5, 1.0, 1e-9 if not lsm else 1e-12
    ref = orc.project(f["p"], f["u"], f["v"], f["w"], f["us"], f["vs"], f["ws"], dt, alfapr,
                      dens=f["dens"] if lsm else None, tol=eps, maxcy=60, stop_rule=1)
    hp, hu, hv, hw = (to_host(blocks, f[k]) for k in ("p", "u", "v", "w"))
    info = s.project(hp, hu, hv, hw, to_host(blocks, f["us"]), to_host(blocks, f["vs"]), to_host(blocks, f["ws"]),
                     dt, alfapr, tol=eps, maxcy=60, stop_rule=1, history=True)
    assert info["outer"] == ref["cycles"], (info["outer"], ref["cycles"])
    assert info["converged"] == (ref["status"] == 0)
    np.testing.assert_array_equal(info["history"], ref["history"])
    for ib, d in enumerate(blocks):
        gp = _canon(h3d, hp[ib], d)
        m = _face_mask(gp)
        assert np.array_equal(gp[m], ref["p"][ib][m]), ib
        for name, hh in (("u", hu), ("v", hv), ("w", hw)):
            assert np.array_equal(_canon(h3d, hh[ib], d), ref[name][ib]), (name, ib)
    s.close()


@pytest.mark.parametrize("layout", [LAYOUTS[1], LAYOUTS[3]])
def test_projection_relative_rule_and_resident_fields(oracle_mod, h3d, layout):
    """stop_rule 0 (||su|| <= tol ||su_0||) on the resident fields: cycles
    equal, history within rounding of the norms, su left in field 'b'."""
    blocks, s, orc, f = _pair(oracle_mod, h3d, layout)
    ref = orc.project(f["p"], f["u"], f["v"], f["w"], f["us"], f["vs"], f["ws"], 1.0, tol=1e-8, maxcy=80,
                      stop_rule=0)
    _upload_all(s, blocks, f)
    info = s.project_resident(1.0, tol=1e-8, maxcy=80, stop_rule=0, history=True)
    assert info["converged"] and info["outer"] == ref["cycles"]
    np.testing.assert_allclose(info["history"], ref["history"], rtol=1e-10, atol=0)
    su_last, _, _ = orc.calmas(ref["u"], ref["v"], ref["w"], 1.0)
    for ib, d in enumerate(blocks):
        host = h3d.host_field(d)
        s.download("b", ib, host)
        assert np.array_equal(h3d.interior(host, d), su_last[ib])
    s.close()


@pytest.mark.parametrize("layout", [LAYOUTS[1], LAYOUTS[3]])
def test_projection_mixed_precision(oracle_mod, h3d, layout):
    """FP32 V-cycles inside the FP64 projection loop converge to the
    tolerance, and the pressure is as close to the FP64 solution (the
    oracle's to 1e-13) as the oracle's own FP64 projection stopped at the
    same tolerance: random face velocities give a divergence dominated by
    short waves, so ||su|| / ||su_0|| = 1e-10 still leaves about 2e-6 of
    relative error in the long waves of p, FP64 or not."""
    blocks, s, orc, f = _pair(oracle_mod, h3d, layout, precision="mixed", coarse_sweeps=16)
    ref = orc.project(f["p"], f["u"], f["v"], f["w"], f["us"], f["vs"], f["ws"], 1.0, tol=1e-13, maxcy=400,
                      stop_rule=0)
    same = orc.project(f["p"], f["u"], f["v"], f["w"], f["us"], f["vs"], f["ws"], 1.0, tol=1e-10, maxcy=400,
                       stop_rule=0)
    assert ref["status"] == 0 and same["status"] == 0
    hp, hu, hv, hw = (to_host(blocks, f[k]) for k in ("p", "u", "v", "w"))
    info = s.project(hp, hu, hv, hw, to_host(blocks, f["us"]), to_host(blocks, f["vs"]), to_host(blocks, f["ws"]),
                     1.0, tol=1e-10, maxcy=200, stop_rule=0)
    assert info["converged"] and info["relres"] <= 1e-10
    want = [x[1:-1, 1:-1, 1:-1] for x in ref["p"]]
    got = [h3d.interior(x, d) for x, d in zip(hp, blocks)]
    e_fp64 = mean_removed_rel([x[1:-1, 1:-1, 1:-1] for x in same["p"]], want)
    e_mixed = mean_removed_rel(got, want)
    assert e_mixed <= 2.0 * e_fp64 + 1e-12, (e_mixed, e_fp64)
    s.close()


def test_projection_config2_geometry(oracle_mod, h3d):
    """192^3 as 2x2x2 blocks of 96^3, periodic in x, 6 levels (the geometry
    of the configuration-2 workload), FP64 against the oracle bit for bit
    under the reference stop rule."""
    layout = ((2, 2, 2), (96, 96, 96), [P, P, W, W, W, W], 6)
    blocks, s, orc, f = _pair(oracle_mod, h3d, layout, seed=1002)
    import oracle.oracle as O  # noqa: F401  (threads for the large case)
    O.lib().or_set_threads(16)
    zero = [np.zeros_like(x) for x in f["p"]]
    eps = 1e-11
    ref = orc.project(zero, f["u"], f["v"], f["w"], f["us"], f["vs"], f["ws"], 1.0, tol=eps, maxcy=100, stop_rule=1)
    hp = to_host(blocks, zero)
    hu, hv, hw = (to_host(blocks, f[k]) for k in ("u", "v", "w"))
    info = s.project(hp, hu, hv, hw, to_host(blocks, f["us"]), to_host(blocks, f["vs"]), to_host(blocks, f["ws"]),
                     1.0, tol=eps, maxcy=100, stop_rule=1, history=True)
    O.lib().or_set_threads(1)
    assert ref["status"] == 0 and info["converged"]
    assert info["outer"] == ref["cycles"]
    np.testing.assert_array_equal(info["history"], ref["history"])
    for ib, d in enumerate(blocks):
        gp = _canon(h3d, hp[ib], d)
        m = _face_mask(gp)
        assert np.array_equal(gp[m], ref["p"][ib][m]), ib
        assert np.array_equal(_canon(h3d, hu[ib], d), ref["u"][ib]), ib
    s.close()
