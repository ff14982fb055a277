"""Local mesh refinement (LMR = 2): blocks of refinement ratio rdiv next to
blocks of ratio rdiv/2 or 2 rdiv (localparameters.for:24-59; exchangepp.for
LMR branches :164-189, :447-458, :652-700, :2115-2131).

CPU: the library's expression form of each level's fill, applied in FP64,
equals the oracle's mgbound + exchangepp cell for cell (ghost corners and
edges included), and on equal-resolution layouts it is the gather table.
GPU: V-cycles and solves of LMR layouts against the oracle (the mgkcyc
golden fixtures of the reference's own Fortran are in test_golden.py).
"""
import numpy as np
import pytest

from tests.helpers import apply_expr, to_oracle_descs

W, P = 4, 5


def lmr_layout(name):
    """(descs, ngrd_gl) of a named LMR layout (product descriptors)."""
    from hydro3d_b200 import topology as T
    layouts = {
        # name: (blocks per axis, cells per block (unrefined), bc, ngrid_input, rdiv, h)
        "walls_2x1x1": ((2, 1, 1), (8, 8, 8), [W] * 6, 3, [1, 2]),
        "corners_2x2x2": ((2, 2, 2), (8, 8, 8), [W] * 6, 3, [2, 1, 1, 1, 1, 1, 1, 1]),
        "diag_2x2x2": ((2, 2, 2), (8, 8, 8), [W] * 6, 3, [2, 1, 1, 1, 1, 1, 1, 2]),
        "periodic_x_1x2x2": ((1, 2, 2), (8, 8, 8), [P, P, W, W, W, W], 2, [1, 2, 2, 1]),
        "ratio4_2x2x1": ((2, 2, 1), (4, 4, 4), [W, W, W, W, P, P], 2, [2, 2, 2, 4]),
        "strip_3x1x1": ((3, 1, 1), (8, 4, 4), [W, W, P, P, W, W], 2, [1, 2, 1]),
    }
    nb, n, bc, ngi, rdiv = layouts[name]
    descs = T.block_grid(nb, n, bc, (1.0 / 32,) * 3, ngi)
    T.refine(descs, rdiv, ngi)
    return descs, ngi + max(r.bit_length() - 1 for r in rdiv)


LAYOUTS = ["walls_2x1x1", "corners_2x2x2", "diag_2x2x2", "periodic_x_1x2x2", "ratio4_2x2x1", "strip_3x1x1"]


def _level_dims(d, g):
    gl = min(g, d.ngrid)
    s = 2 ** (gl - 1)
    return d.n[2] // s, d.n[1] // s, d.n[0] // s


@pytest.mark.parametrize("name", LAYOUTS)
def test_expr_fill_matches_oracle(h3d, oracle_mod, name):
    """Every level, kinds 0 (mgbound + exchangepp) and 1 (exchangepp): the
    expression table applied to random level arrays gives the oracle's
    result bit for bit on every cell."""
    descs, ngrd = lmr_layout(name)
    od = to_oracle_descs(oracle_mod, descs)
    orc = oracle_mod.Oracle(od, ngrd)
    orc.coeff()
    rng = np.random.default_rng(5)
    lmr_levels = 0
    for g in range(1, ngrd + 1):
        for kind in (0, 1):
            arrs = []
            for ib, d in enumerate(descs):
                nz, ny, nx = _level_dims(d, g)
                a = rng.standard_normal((nz + 2, ny + 2, nx + 2))
                arrs.append(a)
                orc.put_phi(g, ib, a)
            if kind == 0:
                orc.mgbound(g)
            orc.exchangepp(g)
            nodes, dst, src = h3d.mg.halo_expr(descs, g, kind)
            lmr_levels += int(len(nodes) > 0 and (nodes[:, 0] != 0).any())
            flat = apply_expr(nodes, dst, src, np.concatenate([a.ravel() for a in arrs]))
            off = 0
            for ib, a in enumerate(arrs):
                mine = flat[off:off + a.size].reshape(a.shape)
                off += a.size
                ref = orc.get_phi(g, ib)
                assert np.array_equal(mine, ref), (name, g, kind, ib, np.argwhere(mine != ref)[:5].tolist())
    orc.close()
    assert lmr_levels > 0


@pytest.mark.parametrize("layout", [((2, 2, 2), [W] * 6), ((2, 1, 3), [P] * 6), ((3, 2, 1), [W, W, P, P, W, W])])
def test_expr_fill_is_the_gather_at_equal_resolution(h3d, layout):
    """Without refinement the expression table has copy nodes only (reads of
    pre-fill ghosts) and, resolved, is the gather table h3d_halo_table gives."""
    from hydro3d_b200 import topology as T
    nb, bc = layout
    descs = T.block_grid(nb, (8, 8, 8), bc, (1.0 / 32,) * 3, 3)
    for g in (1, 2, 3):
        for kind in (0, 1, 2):
            nodes, dst, src = h3d.mg.halo_expr(descs, g, kind)
            gd, gs = h3d.halo_table(descs, g, kind)
            assert (nodes[:, 0] == 0).all() if len(nodes) else True
            res = src.copy()
            isnode = (src >> 30) == 1
            res[isnode] = nodes[src[isnode] & 0x3FFFFFFF, 1]
            assert np.array_equal(dst, gd) and np.array_equal(res, gs), (nb, g, kind)


def test_rejects_refinement_jumps_of_four(h3d):
    """Face neighbours of ratios 1 and 4: the reference's branches assume a
    factor of 2 (exchangepp.for:164-189)."""
    from hydro3d_b200 import topology as T
    descs = T.block_grid((2, 1, 1), (4, 4, 4), [W] * 6, (1.0 / 32,) * 3, 2)
    T.refine(descs, [1, 4], 2)
    with pytest.raises(h3d.H3DError):
        h3d.mg.halo_expr(descs, 1, 0)


# --------------------------------------------------------------------- GPU
def _host_fields(h3d, descs, canon_interior):
    out = []
    for d, a in zip(descs, canon_interior):
        x = h3d.host_field(d)
        h3d.interior(x, d)[...] = a
        out.append(x)
    return out


def _manufactured(oracle_mod, descs, ngrd, seed):
    """b = A p for a random p (A: the level-1 operator with the LMR ghost
    fill, as the oracle's residual applies it), so b is in A's range."""
    orc = oracle_mod.Oracle(to_oracle_descs(oracle_mod, descs), ngrd)
    orc.coeff()
    rng = np.random.default_rng(seed)
    pex = [rng.standard_normal((d.n[2] + 2, d.n[1] + 2, d.n[0] + 2)) for d in descs]
    zeros = [np.zeros((d.n[2], d.n[1], d.n[0])) for d in descs]
    r, _, _, _ = orc.residual(pex, zeros)
    return orc, [-x for x in r]


@pytest.mark.gpu
@pytest.mark.parametrize("name", LAYOUTS)
@pytest.mark.parametrize("itr", [3, 2])
def test_lmr_vcycle_bitexact(h3d, oracle_mod, name, itr):
    """Two V-cycles (mgkcyc) in FP64 on an LMR layout equal the oracle's bit
    for bit, ghosts included (red-black GS and line TDMA smoothers)."""
    descs, ngrd = lmr_layout(name)
    for d in descs:
        d.pl = 1
        for a in range(3):
            d.ttc[a] = d.n[a] + 2
    rng = np.random.default_rng(17)
    pp = [rng.standard_normal((d.n[2] + 2, d.n[1] + 2, d.n[0] + 2)) for d in descs]
    su_c = [rng.standard_normal((d.n[2], d.n[1], d.n[0])) for d in descs]
    orc = oracle_mod.Oracle(to_oracle_descs(oracle_mod, descs), ngrd, mg_itrsch=itr)
    orc.coeff()
    want = [a.copy() for a in pp]
    for _ in range(2):
        want = orc.mgkcyc(want, su_c)
    s = h3d.MultigridSolver(descs, ngrd, mg_itrsch=itr)
    su = _host_fields(h3d, descs, su_c)
    got = [a.copy() for a in pp]
    for _ in range(2):
        s.mgkcyc(got, su)
    for ib in range(len(descs)):
        assert np.array_equal(got[ib], want[ib]), (name, ib, float(np.abs(got[ib] - want[ib]).max()))
    s.close()
    orc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["walls_2x1x1", "corners_2x2x2", "periodic_x_1x2x2", "ratio4_2x2x1"])
def test_lmr_newsolv_matches_oracle(h3d, oracle_mod, name):
    """newsolv_mg (FP64 defect correction) on an LMR layout: the same cycle
    count and residual history as the oracle's solve (the norms are summed in
    different orders: equal to 1e-14 of ||b||), the same pressure."""
    from tests.helpers import interior_of_host, mean_removed_rel
    descs, ngrd = lmr_layout(name)
    orc, b_c = _manufactured(oracle_mod, descs, ngrd, 23)
    ref = orc.solve([np.zeros((d.n[2] + 2, d.n[1] + 2, d.n[0] + 2)) for d in descs], b_c, tol=1e-10, maxcy=200)
    s = h3d.MultigridSolver(descs, ngrd)
    b = _host_fields(h3d, descs, b_c)
    p = [h3d.host_field(d) for d in descs]
    info = s.newsolv_mg(p, b, tol=1e-10, maxcy=200, history=True)
    assert ref["status"] == 0 and info["converged"], (ref["status"], info)
    assert info["cycles"] == ref["cycles"]
    np.testing.assert_allclose(info["history"], ref["history"], rtol=1e-8, atol=1e-14)
    got = [interior_of_host(x, d) for x, d in zip(p, descs)]
    want = [x[1:-1, 1:-1, 1:-1] for x in ref["p"]]
    assert mean_removed_rel(got, want) <= 1e-9
    s.close()
    orc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["walls_2x1x1", "corners_2x2x2", "periodic_x_1x2x2"])
def test_lmr_mixed_precision(h3d, oracle_mod, name):
    """FP32 V-cycles inside FP64 refinement on an LMR layout reach 1e-11 and
    agree with the oracle's FP64 solution (to 1e-12) to 1e-8."""
    from tests.helpers import interior_of_host, mean_removed_rel
    descs, ngrd = lmr_layout(name)
    orc, b_c = _manufactured(oracle_mod, descs, ngrd, 29)
    ref = orc.solve([np.zeros((d.n[2] + 2, d.n[1] + 2, d.n[0] + 2)) for d in descs], b_c, tol=1e-12, maxcy=300)
    s = h3d.MultigridSolver(descs, ngrd, precision="mixed")
    b = _host_fields(h3d, descs, b_c)
    p = [h3d.host_field(d) for d in descs]
    info = s.newsolv_mg(p, b, tol=1e-11, maxcy=400)
    assert info["converged"] and info["relres"] <= 1e-11, info
    got = [interior_of_host(x, d) for x, d in zip(p, descs)]
    want = [x[1:-1, 1:-1, 1:-1] for x in ref["p"]]
    assert mean_removed_rel(got, want) <= 1e-8
    s.close()
    orc.close()


@pytest.mark.gpu
def test_lmr_exchangepp_entry_point(h3d, oracle_mod):
    """h3d_mg_exchangepp on a level with refinement interfaces applies the
    expression fill: the oracle's exchangepp bit for bit."""
    descs, ngrd = lmr_layout("corners_2x2x2")
    orc = oracle_mod.Oracle(to_oracle_descs(oracle_mod, descs), ngrd)
    orc.coeff()
    s = h3d.MultigridSolver(descs, ngrd)
    s.coeff()
    rng = np.random.default_rng(3)
    for g in (1, 2):
        arrs = []
        for ib, d in enumerate(descs):
            nz, ny, nx = _level_dims(d, g)
            a = rng.standard_normal((nz + 2, ny + 2, nx + 2))
            arrs.append(a)
            orc.put_phi(g, ib, a)
            s.put_level(g, "phi", ib, a)
        orc.exchangepp(g)
        s.exchangepp(g)
        for ib in range(len(descs)):
            assert np.array_equal(s.get_level(g, "phi", ib), orc.get_phi(g, ib)), (g, ib)
    s.close()
    orc.close()


def test_lmr_rejections(h3d):
    """What the drop-in refuses with refinement: L_LSM coefficients, periodic
    partners of different ratio, level counts that do not follow rdiv."""
    from hydro3d_b200 import topology as T
    bad_config = h3d._lib.H3D_ERR_BAD_CONFIG  # checked before any device call
    descs, ngrd = lmr_layout("walls_2x1x1")
    with pytest.raises(h3d.H3DError) as e:
        h3d.MultigridSolver(descs, ngrd, var_coef=True)
    assert e.value.code == bad_config
    bad = T.block_grid((2, 1, 1), (8, 8, 8), [P, P, W, W, W, W], (1.0 / 32,) * 3, 3)
    T.refine(bad, [1, 2], 3)
    with pytest.raises(h3d.H3DError) as e:
        h3d.MultigridSolver(bad, 4)
    assert e.value.code == bad_config
    descs[1].ngrid = 3
    with pytest.raises(h3d.H3DError) as e:
        h3d.MultigridSolver(descs, ngrd)
    assert e.value.code == bad_config
