"""CPU checks of the oracle's projection (calvel, calmas, exchange(1..3),
newsolv_mg with velocities; press.for:2-207, newsolv_mg.for:2-93).

The golden fixtures (tests/test_golden.py) pin the restatement against the
reference's own press.for / exchange.for run by the translator; these are
properties on top: with p = 0 calvel copies ustar onto the faces the
reference updates and calmas is the discrete divergence of the staggered
field (computed independently in numpy); the converged projection leaves a
divergence-free velocity whose pressure agrees with the defect-correction
solve of b = div(ustar)/dt; the face ghosts hold the neighbour's adjacent
face.
"""
import numpy as np
import pytest

from tests.helpers import mean_removed_rel, projection_fields, to_oracle_descs

W, P = 4, 5
LAYOUTS = [
    ((1, 1, 1), (16, 16, 16), [W] * 6, 3),
    ((2, 2, 1), (8, 16, 8), [P, P, W, W, W, W], 3),
    ((2, 1, 2), (8, 8, 8), [P] * 6, 3),
]


def _setup(O, layout, lsm=False, seed=5):
    from hydro3d_b200 import topology
    nblk, n, bc, ngrid = layout
    blocks = topology.block_grid(nblk, n, bc, [1.0 / 32] * 3, ngrid, resolve=O.topology)
    orc = O.Oracle(to_oracle_descs(O, blocks), ngrid, 3, 2, 1, lsm=lsm)
    f = projection_fields(blocks, seed, lsm)
    if lsm:
        for ib, (d, x) in enumerate(zip(blocks, f["dens"])):
            orc.set_density(ib, x[1:-1, 1:-1, 1:-1])
    orc.coeff()
    return blocks, orc, f


def _numpy_div(u, v, w, h):
    return ((u[1:-1, 1:-1, 1:-1] - u[1:-1, 1:-1, :-2]) / h[0] + (v[1:-1, 1:-1, 1:-1] - v[1:-1, :-2, 1:-1]) / h[1]
            + (w[1:-1, 1:-1, 1:-1] - w[:-2, 1:-1, 1:-1]) / h[2])


@pytest.mark.parametrize("layout", LAYOUTS)
def test_calvel_with_zero_pressure_copies_ustar(oracle_mod, layout):
    blocks, orc, f = _setup(oracle_mod, layout)
    zero = [np.zeros_like(x) for x in f["p"]]
    u, v, w = orc.calvel(f["u"], f["v"], f["w"], f["us"], f["vs"], f["ws"], zero, dt=0.5)
    for ib, d in enumerate(blocks):
        nx, ny, nz = d.n
        wall_e = d.nb_face[1] < 0 and d.bc[1] != 5
        xe = nx - 1 if wall_e else nx
        np.testing.assert_array_equal(u[ib][1:-1, 1:-1, 1:xe + 1], f["us"][ib][1:-1, 1:-1, 1:xe + 1])
        if wall_e:  # the wall face keeps its boundary value
            np.testing.assert_array_equal(u[ib][1:-1, 1:-1, nx], f["u"][ib][1:-1, 1:-1, nx])
        # face ghosts of the interior rows come from the source's adjacent face
        src = d.nb_face[0] if d.nb_face[0] >= 0 else (
            (ib if d.nb_face[1] < 0 else d.nb_periodic[0]) if d.bc[0] == 5 else -1)
        if src >= 0:
            s = blocks[src]
            np.testing.assert_array_equal(u[ib][1:-1, 1:-1, 0], u[src][1:-1, 1:-1, s.n[0]])
        else:
            np.testing.assert_array_equal(u[ib][1:-1, 1:-1, 0], f["u"][ib][1:-1, 1:-1, 0])
        # edge rows of the ghost faces are not written
        np.testing.assert_array_equal(u[ib][0, :, 0], f["u"][ib][0, :, 0])


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("lsm", [False, True])
def test_calmas_is_the_staggered_divergence(oracle_mod, layout, lsm):
    blocks, orc, f = _setup(oracle_mod, layout, lsm)
    dt = 0.25
    su, ss, rmax = orc.calmas(f["u"], f["v"], f["w"], dt)
    want_max = 0.0
    for ib, d in enumerate(blocks):
        h = d.h
        div = _numpy_div(f["u"][ib], f["v"][ib], f["w"][ib], h)
        want = div * h[0] * h[1] * h[2] / dt if lsm else div / dt
        np.testing.assert_array_equal(su[ib], want)
        want_max = max(want_max, float(np.abs(div * h[0] * h[1] * h[2]).max()))
    assert rmax == want_max
    assert np.isclose(ss, sum(float((x * x).sum()) for x in su), rtol=1e-13)


@pytest.mark.parametrize("layout", LAYOUTS)
def test_projection_converges_to_the_defect_correction_solution(oracle_mod, layout):
    """dt = alfapr = 1 from p = 0: su = div(ustar) - A p, so the projection's
    p solves A p = div(ustar) like or_solve; the final u is divergence free."""
    blocks, orc, f = _setup(oracle_mod, layout)
    zero = [np.zeros_like(x) for x in f["p"]]
    res = orc.project(zero, f["u"], f["v"], f["w"], f["us"], f["vs"], f["ws"], dt=1.0, tol=1e-10, maxcy=200,
                      stop_rule=0)
    assert res["status"] == 0
    # residual divergence of the returned velocity
    su, ss, rmax = orc.calmas(res["u"], res["v"], res["w"], 1.0)
    su0, ss0, _ = orc.calmas(*orc.calvel(f["u"], f["v"], f["w"], f["us"], f["vs"], f["ws"], zero, 1.0), 1.0)
    assert np.sqrt(ss) <= 1e-10 * np.sqrt(ss0) * 1.0001
    # the same pressure from the defect-correction solve of A p = div(ustar)
    ref = orc.solve(zero, su0, tol=1e-10, maxcy=200)
    assert ref["status"] == 0
    got = [x[1:-1, 1:-1, 1:-1] for x in res["p"]]
    want = [x[1:-1, 1:-1, 1:-1] for x in ref["p"]]
    assert mean_removed_rel(got, want) < 1e-8


def test_projection_reference_stop_rule(oracle_mod):
    """stop_rule 1 (newsolv_mg.for:57): stops at the first cycle after the
    second whose rmax is below eps; history holds rmax."""
    blocks, orc, f = _setup(oracle_mod, LAYOUTS[1])
    zero = [np.zeros_like(x) for x in f["p"]]
    res = orc.project(zero, f["u"], f["v"], f["w"], f["us"], f["vs"], f["ws"], dt=1.0, tol=1e-9, maxcy=200,
                      stop_rule=1)
    assert res["status"] == 0 and res["cycles"] >= 2
    hist = res["history"]
    assert hist[-1] < 1e-9 and res["rmax"] == hist[-1]
    assert all(x >= 1e-9 for x in hist[1:-1]) or res["cycles"] == 2
