"""GPU parity: every reference routine on the CUDA path vs the oracle.

The FP64 path is compared bit for bit (the library is built without FMA
contraction and follows the reference's operand order); the FP32 path of the
mixed-precision solver is compared with a relative tolerance of 2e-5.
All calls go through the C ABI (hydro3d_b200 -> libh3dmg.so).
"""
import numpy as np
import pytest

from tests.helpers import mean_removed_rel, to_oracle_descs

pytestmark = pytest.mark.gpu

W, P = 4, 5
LAYOUTS = [
    ((1, 1, 1), (16, 16, 16), [W] * 6, 3),
    ((2, 2, 2), (8, 16, 8), [P, P, W, W, W, W], 3),
    ((3, 2, 2), (16, 8, 8), [W, W, P, P, W, W], 2),
    ((2, 1, 3), (8, 8, 16), [P] * 6, 3),
    # more blocks than one thread-block cluster holds: the single-CTA coarse tail
    ((3, 3, 2), (8, 8, 8), [P, P, W, W, W, W], 3),
]
FP32_RTOL = 2e-5


def _pair(O, h3d, layout, precision="fp64", var=False, use_graph=False, itrsch=3):
    nblk, n, bc, ngrid = layout
    blocks = h3d.topology.block_grid(nblk, n, bc, [1.0 / 32] * 3, ngrid)
    s = h3d.MultigridSolver(blocks, ngrid, mg_itrsch=itrsch, precision=precision, var_coef=var, use_graph=use_graph)
    orc = O.Oracle(to_oracle_descs(O, blocks), ngrid, itrsch, 2, 1, lsm=var)
    return blocks, s, orc


def _rand_level(rng, s, orc, g, fields=("phi", "rhs")):
    for ib in range(len(s.blocks)):
        nz, ny, nx = s.level_dims(g, ib)
        if "phi" in fields:
            a = rng.standard_normal((nz + 2, ny + 2, nx + 2))
            s.put_level(g, "phi", ib, a)
            orc.put_phi(g, ib, a)
        if "rhs" in fields:
            r = rng.standard_normal((nz, ny, nx))
            s.put_level(g, "rhs", ib, r)
            orc.put_rhs(g, ib, r)


def _assert_level(s, orc, g, field="phi", exact=True):
    for ib in range(len(s.blocks)):
        a = s.get_level(g, field, ib)
        b = orc.get_phi(g, ib) if field == "phi" else orc.get_rhs(g, ib)
        if exact:
            assert np.array_equal(a, b), (g, ib, float(np.abs(a - b).max()))
        else:
            np.testing.assert_allclose(a, b, rtol=FP32_RTOL, atol=FP32_RTOL * np.abs(b).max())


@pytest.mark.parametrize("layout", LAYOUTS)
def test_mgrelax_bitexact(oracle_mod, h3d, layout):
    blocks, s, orc = _pair(oracle_mod, h3d, layout)
    s.coeff(); orc.coeff()
    rng = np.random.default_rng(1)
    for g in range(1, layout[3] + 1):
        _rand_level(rng, s, orc, g)
        s.mgrelax(g, 2)
        orc.mgrelax(g, 2)
        _assert_level(s, orc, g)
    s.close()


@pytest.mark.parametrize("layout", LAYOUTS)
def test_mgrestr_mgcorr_bitexact(oracle_mod, h3d, layout):
    blocks, s, orc = _pair(oracle_mod, h3d, layout)
    s.coeff(); orc.coeff()
    rng = np.random.default_rng(2)
    for g in range(2, layout[3] + 1):
        _rand_level(rng, s, orc, g - 1)
        s.mgrestr(g)
        orc.mgrestr(g)
        _assert_level(s, orc, g, "rhs")
        _assert_level(s, orc, g, "phi")
        _rand_level(rng, s, orc, g, ("phi",))
        _rand_level(rng, s, orc, g - 1, ("phi",))
        s.mgcorr(g - 1)
        orc.mgcorr(g - 1)
        _assert_level(s, orc, g - 1)
    s.close()


@pytest.mark.parametrize("layout", LAYOUTS)
def test_mgbound_exchangepp_bitexact(oracle_mod, h3d, layout):
    blocks, s, orc = _pair(oracle_mod, h3d, layout)
    s.coeff(); orc.coeff()
    rng = np.random.default_rng(3)
    _rand_level(rng, s, orc, 1)
    s.mgbound(1); orc.mgbound(1)
    _assert_level(s, orc, 1)
    _rand_level(rng, s, orc, 2)
    s.exchangepp(2); orc.exchangepp(2)
    _assert_level(s, orc, 2)
    s.close()


@pytest.mark.parametrize("layout", LAYOUTS)
def test_vcycle_bitexact(oracle_mod, h3d, layout):
    blocks, s, orc = _pair(oracle_mod, h3d, layout)
    s.coeff(); orc.coeff()
    rng = np.random.default_rng(4)
    _rand_level(rng, s, orc, 1)
    s.vcycle(); orc.vcycle()
    _assert_level(s, orc, 1)
    s.vcycle(); orc.vcycle()
    _assert_level(s, orc, 1)
    s.close()


def test_var_coef_bitexact(oracle_mod, h3d):
    layout = ((2, 1, 2), (16, 16, 8), [W] * 6, 3)
    blocks, s, orc = _pair(oracle_mod, h3d, layout, var=True)
    rng = np.random.default_rng(5)
    for ib, d in enumerate(blocks):
        dens = h3d.host_field(d)
        rho = np.exp(rng.uniform(0, np.log(1000.0), (d.n[2], d.n[1], d.n[0])))
        h3d.interior(dens, d)[...] = rho
        s.set_density(ib, dens)
        orc.set_density(ib, rho)
    s.coeff(); orc.coeff()
    for g in (1, 2, 3):
        _rand_level(rng, s, orc, g)
        s.mgrelax(g, 1); orc.mgrelax(g, 1)
        _assert_level(s, orc, g)
    _rand_level(rng, s, orc, 1)
    s.mgrestr(2); orc.mgrestr(2)
    _assert_level(s, orc, 2, "rhs")
    _rand_level(rng, s, orc, 1)
    s.vcycle(); orc.vcycle()
    _assert_level(s, orc, 1)
    s.close()


def test_fp32_kernels_close(oracle_mod, h3d):
    layout = ((2, 2, 1), (16, 16, 16), [P, P, W, W, W, W], 3)
    blocks, s, orc = _pair(oracle_mod, h3d, layout, precision="mixed")
    s.coeff(); orc.coeff()
    rng = np.random.default_rng(6)
    _rand_level(rng, s, orc, 1)
    s.mgrelax(1, 2); orc.mgrelax(1, 2)
    _assert_level(s, orc, 1, exact=False)
    _rand_level(rng, s, orc, 1)
    s.mgrestr(2); orc.mgrestr(2)
    _assert_level(s, orc, 2, "rhs", exact=False)
    s.close()


@pytest.mark.parametrize("layout", [((4, 2, 2), (16, 16, 16), [P, P, W, W, W, W], 4),
                                    ((3, 3, 2), (8, 8, 8), [W, W, P, P, W, W], 3)])
def test_mixed_vcycle_coarse_tails(oracle_mod, h3d, layout):
    """Mixed-precision V-cycles whose coarse levels run fused: 16 equal blocks
    (one thread-block cluster) and 18 blocks (one CTA), against the FP64
    oracle V-cycle; tolerance 1e-4 of the largest value.  Coarse levels are
    read back too (the fused tail stores them)."""
    blocks, s, orc = _pair(oracle_mod, h3d, layout, precision="mixed")
    s.coeff(); orc.coeff()
    rng = np.random.default_rng(31)
    _rand_level(rng, s, orc, 1)
    for _ in range(2):
        s.vcycle(); orc.vcycle()
        for ib in range(len(blocks)):
            a, b = s.get_level(1, "phi", ib), orc.get_phi(1, ib)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-4 * np.abs(b).max())
    g = layout[3]
    for ib in range(len(blocks)):
        a, b = s.get_level(g - 1, "rhs", ib), orc.get_rhs(g - 1, ib)
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-4 * np.abs(b).max())
    s.close()


def _host_problem(h3d, blocks, seed, pl):
    rng = np.random.default_rng(seed)
    b, p, bc_, pc_ = [], [], [], []
    for d in blocks:
        bh = h3d.host_field(d)
        bi = rng.standard_normal((d.n[2], d.n[1], d.n[0]))
        h3d.interior(bh, d)[...] = bi
        b.append(bh)
        p.append(h3d.host_field(d))
    # wall and periodic faces only: the operator is singular, the rhs must have zero mean
    m = np.mean(np.concatenate([h3d.interior(x, d).ravel() for x, d in zip(b, blocks)]))
    for x, d in zip(b, blocks):
        h3d.interior(x, d)[...] -= m
    return b, p


@pytest.mark.parametrize("layout", [((1, 1, 1), (32, 32, 32), [W] * 6, 4),
                                    ((2, 2, 2), (16, 16, 16), [P, P, W, W, W, W], 4)])
def test_newsolv_matches_oracle(oracle_mod, h3d, layout):
    nblk, n, bc, ngrid = layout
    blocks = h3d.topology.block_grid(nblk, n, bc, [1.0 / 32] * 3, ngrid, pl=2)
    b, p = _host_problem(h3d, blocks, 11, 2)
    s = h3d.MultigridSolver(blocks, ngrid)
    info = s.newsolv_mg(p, b, tol=1e-8, maxcy=300, history=True)
    orc = oracle_mod.Oracle(to_oracle_descs(oracle_mod, blocks), ngrid)
    orc.coeff()
    from tests.helpers import canon_from_host, interior_of_host
    ref = orc.solve([np.zeros((d.n[2] + 2, d.n[1] + 2, d.n[0] + 2)) for d in blocks],
                    [interior_of_host(x, d) for x, d in zip(b, blocks)], tol=1e-8, maxcy=300)
    assert info["converged"] and ref["status"] == 0
    assert abs(info["cycles"] - ref["cycles"]) <= 2
    got = [interior_of_host(x, d) for x, d in zip(p, blocks)]
    want = [x[1:-1, 1:-1, 1:-1] for x in ref["p"]]
    assert mean_removed_rel(got, want) <= 1e-7
    np.testing.assert_allclose(info["history"], ref["history"], rtol=1e-9, atol=0)
    s.close()


def test_newsolv_wide_ragged_rows(oracle_mod, h3d):
    """Twelve outer iterations of newsolv_mg on blocks of 96 x 12 x 8 cells
    (rows of 48 cell pairs, row tiles of the defect that end inside a block,
    several plane chunks per block) against the oracle: residual history
    within 1e-9, iterate within 1e-10 (the two sum the norms in different
    orders).  The elongated blocks converge slowly, so no convergence is
    asked for."""
    blocks = h3d.topology.block_grid((1, 2, 1), (96, 12, 8), [W, W, P, P, W, W], [1.0 / 32] * 3, 3, pl=2)
    b, p = _host_problem(h3d, blocks, 16, 2)
    s = h3d.MultigridSolver(blocks, 3)
    info = s.newsolv_mg(p, b, tol=1e-30, maxcy=12, history=True)
    orc = oracle_mod.Oracle(to_oracle_descs(oracle_mod, blocks), 3)
    orc.coeff()
    from tests.helpers import interior_of_host
    ref = orc.solve([np.zeros((d.n[2] + 2, d.n[1] + 2, d.n[0] + 2)) for d in blocks],
                    [interior_of_host(x, d) for x, d in zip(b, blocks)], tol=1e-30, maxcy=12)
    assert info["cycles"] == ref["cycles"] == 12
    np.testing.assert_allclose(info["history"], ref["history"], rtol=1e-9, atol=0)
    got = [interior_of_host(x, d) for x, d in zip(p, blocks)]
    want = [x[1:-1, 1:-1, 1:-1] for x in ref["p"]]
    assert mean_removed_rel(got, want) <= 1e-10
    s.close()


def test_mgkcyc_host_fields(oracle_mod, h3d):
    blocks = h3d.topology.block_grid((2, 1, 1), (16, 16, 16), [W] * 6, [1.0 / 32] * 3, 3, pl=3)
    b, _ = _host_problem(h3d, blocks, 12, 3)
    rng = np.random.default_rng(13)
    pp = []
    for d in blocks:
        a = h3d.host_field(d)
        a[...] = rng.standard_normal(a.shape)
        pp.append(a)
    outer = [a.copy() for a in pp]
    s = h3d.MultigridSolver(blocks, 3)
    s.mgkcyc(pp, b)
    orc = oracle_mod.Oracle(to_oracle_descs(oracle_mod, blocks), 3)
    orc.coeff()
    from tests.helpers import canon_from_host, interior_of_host
    got = orc.mgkcyc([canon_from_host(a, d) for a, d in zip(outer, blocks)],
                     [interior_of_host(x, d) for x, d in zip(b, blocks)])
    for a, g, o, d in zip(pp, got, outer, blocks):
        assert np.array_equal(canon_from_host(a, d), g)
        # layers beyond the first ghost layer are untouched
        m = np.ones(a.shape, bool)
        pl = d.pl
        m[pl - 1:pl + d.n[2] + 1, pl - 1:pl + d.n[1] + 1, pl - 1:pl + d.n[0] + 1] = False
        assert np.array_equal(a[m], o[m])
    s.close()


def test_graph_and_eager_identical(h3d):
    blocks = h3d.topology.block_grid((2, 2, 1), (16, 16, 16), [P, P, W, W, W, W], [1.0 / 32] * 3, 4)
    b, p = _host_problem(h3d, blocks, 14, 1)
    out = []
    for g in (True, False):
        s = h3d.MultigridSolver(blocks, 4, use_graph=g)
        pc = [x.copy() for x in p]
        info = s.newsolv_mg(pc, b, tol=1e-9, maxcy=200)
        out.append((pc, info["cycles"]))
        s.close()
    assert out[0][1] == out[1][1]
    for a, c in zip(out[0][0], out[1][0]):
        assert np.array_equal(a, c)


def test_mixed_precision_error_vs_fp64(oracle_mod, h3d):
    blocks = h3d.topology.block_grid((4, 2, 2), (16, 16, 16), [W] * 6, [1.0 / 32] * 3, 5)
    b, p = _host_problem(h3d, blocks, 15, 1)
    orc = oracle_mod.Oracle(to_oracle_descs(oracle_mod, blocks), 5)
    orc.coeff()
    from tests.helpers import interior_of_host
    ref = orc.solve([np.zeros((d.n[2] + 2, d.n[1] + 2, d.n[0] + 2)) for d in blocks],
                    [interior_of_host(x, d) for x, d in zip(b, blocks)], tol=1e-12, maxcy=400)
    s = h3d.MultigridSolver(blocks, 5, precision="mixed")
    pm = [x.copy() for x in p]
    info = s.newsolv_mg(pm, b, tol=1e-12, maxcy=400)
    assert info["converged"] and info["relres"] <= 1e-12
    err = mean_removed_rel([interior_of_host(x, d) for x, d in zip(pm, blocks)],
                           [x[1:-1, 1:-1, 1:-1] for x in ref["p"]])
    assert err <= 1e-8, err
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_smoother_variant(oracle_mod, h3d, precision):
    """Each smoother kernel variant (generic tiles, whole-row tiles, TMA-staged
    row tiles, single-barrier TMA row tiles) and several z-chunks give the
    reference sweep, also with ragged row tiles (ny = 12) and rows longer
    than one lane segment of the two-groups-per-lane sweeps (nx = 64, 96):
    bit-exact in FP64, within the FP32 tolerance in the mixed solver's FP32
    levels."""
    rng = np.random.default_rng(7)
    for layout, need in (((2, 2, 1), (32, 16, 16), [P, P, W, W, W, W], 3), 20), \
                        (((2, 1, 1), (32, 12, 10), [W, W, P, P, W, W], 2), 10), \
                        (((1, 1, 1), (96, 12, 8), [W, W, P, P, W, W], 2), 4), \
                        (((2, 1, 1), (64, 8, 6), [P, P, W, W, W, W], 2), 6):
        blocks, s, orc = _pair(oracle_mod, h3d, layout, precision=precision)
        s.coeff(); orc.coeff()
        _, _, nvar = s.get_smoother(1)
        tried = 0
        for v in range(nvar):
            for zc in (3, 16):
                if not s.set_smoother(1, v, zc):
                    continue
                tried += 1
                _rand_level(rng, s, orc, 1)
                s.mgrelax(1, 2)
                orc.mgrelax(1, 2)
                _assert_level(s, orc, 1, exact=(precision == "fp64"))
        assert tried >= need
        s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_restriction_variant(oracle_mod, h3d, precision):
    """Each restriction kernel variant (plain-load tiles and TMA-staged tiles)
    and several coarse z-chunks give the reference mgrestr, also from a zero
    iterate (the level just restricted into) and with ragged row tiles:
    bit-exact in FP64, within the FP32 tolerance on the mixed solver's FP32
    levels."""
    rng = np.random.default_rng(11)
    exact = precision == "fp64"
    for layout in (((2, 2, 1), (32, 16, 16), [P, P, W, W, W, W], 3),
                   ((2, 1, 1), (32, 24, 12), [W, W, P, P, W, W], 3)):
        blocks, s, orc = _pair(oracle_mod, h3d, layout, precision=precision)
        s.coeff(); orc.coeff()
        _, _, nvar = s.get_restriction(2)
        tried = tma = 0
        for v in range(nvar):
            for zc in (1, 3, 8):
                if not s.set_restriction(2, v, zc):
                    continue
                tried += 1
                tma += v >= 4
                _rand_level(rng, s, orc, 1)
                s.mgrestr(2)
                orc.mgrestr(2)
                _assert_level(s, orc, 2, "rhs", exact=exact)
                if s.set_restriction(3, v, zc):  # from the zero iterate of level 2
                    s.mgrestr(3)
                    orc.mgrestr(3)
                    _assert_level(s, orc, 3, "rhs", exact=exact)
        assert tried >= 12 and tma >= 6
        s.close()


def test_mixed_vcycle_every_level2_smoother(oracle_mod, h3d):
    """A mixed-precision V-cycle (FP32 levels, FP64 coarsest) against the FP64
    oracle V-cycle, with every smoother variant on level 2.  Level 2 starts
    each cycle from the zero iterate left by the restriction, so this runs the
    zero-source sweeps too.  Tolerance: 1e-4 of the largest value."""
    layout = ((2, 2, 1), (32, 32, 32), [P, P, W, W, W, W], 4)
    blocks, s, orc = _pair(oracle_mod, h3d, layout, precision="mixed")
    s.coeff(); orc.coeff()
    _, _, nvar = s.get_smoother(2)
    rng = np.random.default_rng(21)
    tried = 0
    for v in range(nvar):
        if not s.set_smoother(2, v, 5):
            continue
        tried += 1
        _rand_level(rng, s, orc, 1)
        s.vcycle()
        orc.vcycle()
        for ib in range(len(blocks)):
            a, b = s.get_level(1, "phi", ib), orc.get_phi(1, ib)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-4 * np.abs(b).max(), err_msg="variant %d" % v)
    assert tried >= 15
    s.close()


# Lexicographic Gauss-Seidel (mg_itrsch 1) and line TDMA (2): the reference's
# sequential orderings as wavefronts, one CTA per block.
@pytest.mark.parametrize("itrsch", [1, 2])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_sequential_smoothers_bitexact(oracle_mod, h3d, layout, itrsch):
    """mgrelax (two sweeps) on every level and two V-cycles, bit for bit."""
    blocks, s, orc = _pair(oracle_mod, h3d, layout, itrsch=itrsch)
    s.coeff(); orc.coeff()
    rng = np.random.default_rng(40 + itrsch)
    for g in range(1, layout[3] + 1):
        _rand_level(rng, s, orc, g)
        s.mgrelax(g, 2)
        orc.mgrelax(g, 2)
        _assert_level(s, orc, g)
    _rand_level(rng, s, orc, 1)
    for _ in range(2):
        s.vcycle(); orc.vcycle()
        _assert_level(s, orc, 1)
    s.close()


@pytest.mark.parametrize("itrsch", [1, 2])
def test_sequential_smoothers_var_coef_and_ragged(oracle_mod, h3d, itrsch):
    """L_LSM coefficients (density ratio up to 1000) and a block whose three
    axes differ (lines of three lengths, anti-diagonals of unequal sides)."""
    layout = ((2, 1, 1), (24, 8, 16), [W] * 6, 2)
    blocks, s, orc = _pair(oracle_mod, h3d, layout, var=True, itrsch=itrsch)
    rng = np.random.default_rng(50 + itrsch)
    for ib, d in enumerate(blocks):
        dens = h3d.host_field(d)
        rho = np.exp(rng.uniform(0, np.log(1000.0), (d.n[2], d.n[1], d.n[0])))
        h3d.interior(dens, d)[...] = rho
        s.set_density(ib, dens)
        orc.set_density(ib, rho)
    s.coeff(); orc.coeff()
    for g in (1, 2):
        _rand_level(rng, s, orc, g)
        s.mgrelax(g, 1); orc.mgrelax(g, 1)
        _assert_level(s, orc, g)
    _rand_level(rng, s, orc, 1)
    s.vcycle(); orc.vcycle()
    _assert_level(s, orc, 1)
    s.close()


@pytest.mark.parametrize("itrsch", [1, 2])
def test_sequential_smoothers_solve(oracle_mod, h3d, itrsch):
    """newsolv_mg with each sequential smoother: the oracle's cycle count and
    residual history; the mixed-precision solve reaches the tolerance."""
    layout = ((2, 2, 1), (16, 16, 16), [P, P, W, W, W, W], 4)
    blocks = h3d.topology.block_grid(layout[0], layout[1], layout[2], [1.0 / 32] * 3, layout[3])
    b, p = _host_problem(h3d, blocks, 60 + itrsch, 1)
    s = h3d.MultigridSolver(blocks, layout[3], mg_itrsch=itrsch)
    info = s.newsolv_mg([x.copy() for x in p], b, tol=1e-8, maxcy=300, history=True)
    orc = oracle_mod.Oracle(to_oracle_descs(oracle_mod, blocks), layout[3], itrsch, 2, 1)
    orc.coeff()
    from tests.helpers import interior_of_host
    ref = orc.solve([np.zeros((d.n[2] + 2, d.n[1] + 2, d.n[0] + 2)) for d in blocks],
                    [interior_of_host(x, d) for x, d in zip(b, blocks)], tol=1e-8, maxcy=300)
    assert info["converged"] and ref["status"] == 0
    assert info["cycles"] == ref["cycles"]
    np.testing.assert_allclose(info["history"], ref["history"], rtol=1e-9, atol=0)
    s.close()
    m = h3d.MultigridSolver(blocks, layout[3], mg_itrsch=itrsch, precision="mixed")
    info = m.newsolv_mg([x.copy() for x in p], b, tol=1e-8, maxcy=300)
    assert info["converged"] and info["relres"] <= 1e-8
    m.close()


def test_zero_source_stencil_matches_window_sweep(h3d, monkeypatch):
    """The first FP32 sweep from a zero iterate runs as a stencil on the
    right-hand side (launch_rbgs_zero32); with H3D_ZERO_STENCIL=0 the tuned
    TMA sweep kernel runs it in its zero-source mode.  The two evaluate the
    same FP32 operations: V-cycles (level 1 from zero after every defect,
    levels 2.. from zero after every restriction) agree bit for bit, on
    walls, periodic faces and 16 blocks."""
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("H3D_ZERO_STENCIL", flag)
        blocks = h3d.topology.block_grid((4, 2, 2), (32, 16, 24), [P, P, W, W, W, W], [1.0 / 32] * 3, 3)
        b, p = _host_problem(h3d, blocks, 70, 1)
        s = h3d.MultigridSolver(blocks, 3, precision="mixed", coarse_sweeps=16)
        pc = [x.copy() for x in p]
        info = s.newsolv_mg(pc, b, tol=1e-30, maxcy=3)
        out.append((pc, info["history"] if "history" in info else info["relres"]))
        s.close()
    for a, c in zip(out[0][0], out[1][0]):
        assert np.array_equal(a, c)
