"""CPU checks of the oracle (the C restatement of the reference MG path).

The reference ships no golden vectors for this path, so besides the golden
fixtures translated from the reference's own Fortran (test_golden.py) the
oracle is pinned here by properties the reference algorithm must satisfy.
"""
import numpy as np
import pytest

from tests.helpers import mean_removed_rel


def _one_block(O, n, ngrid, bc=(4,) * 6, h=None, itrsch=3, lsm=False):
    h = h or [1.0 / n[0]] * 3
    ext = np.array([[0, n[0], 0, n[1], 0, n[2]]])
    descs = O.topology(ext, bc, h, ngrid)
    return descs, O.Oracle(descs, ngrid, itrsch, 2, 1, lsm=lsm)


def _apply_A(O, orc, p_list, descs):
    """-A p via the oracle residual with b = 0."""
    b = [np.zeros((d.n[2], d.n[1], d.n[0])) for d in descs]
    r, rr, bb, _ = orc.residual(p_list, b)
    return [-x for x in r]


def test_cosine_mode_is_eigenvector(oracle_mod):
    O = oracle_mod
    n = (16, 8, 12)
    descs, orc = _one_block(O, n, 3, h=[1 / 16.0] * 3)
    orc.coeff()
    x = (np.arange(n[0]) + 0.5) / n[0]
    y = (np.arange(n[1]) + 0.5) / n[1]
    z = (np.arange(n[2]) + 0.5) / n[2]
    pe = np.cos(np.pi * 2 * x)[None, None, :] * np.cos(np.pi * y)[None, :, None] * np.cos(np.pi * 3 * z)[:, None, None]
    p = np.zeros((n[2] + 2, n[1] + 2, n[0] + 2))
    p[1:-1, 1:-1, 1:-1] = pe
    Ap = _apply_A(O, orc, [p], descs)[0]
    h2 = (1 / 16.0) ** 2
    lam = sum((2 * np.cos(np.pi * k / m) - 2) / h2 for k, m in ((2, n[0]), (1, n[1]), (3, n[2])))
    np.testing.assert_allclose(Ap, lam * pe, rtol=0, atol=1e-9 * abs(lam))


def test_manufactured_solution(oracle_mod):
    O = oracle_mod
    n = (32, 32, 32)
    descs, orc = _one_block(O, n, 4)
    orc.coeff()
    c = (np.arange(32) + 0.5) / 32
    pe = np.cos(np.pi * c)[None, None, :] * np.cos(2 * np.pi * c)[None, :, None] + np.cos(np.pi * c)[:, None, None]
    pg = np.zeros((34, 34, 34))
    pg[1:-1, 1:-1, 1:-1] = pe
    b = _apply_A(O, orc, [pg], descs)
    res = orc.solve([np.zeros((34, 34, 34))], b, tol=1e-11, maxcy=400)
    assert res["status"] == 0
    assert mean_removed_rel([res["p"][0][1:-1, 1:-1, 1:-1]], [pe]) < 1e-7


def test_constant_in_null_space_and_symmetry(oracle_mod):
    O = oracle_mod
    ext = np.array([[0, 8, 0, 8, 0, 8], [8, 16, 0, 8, 0, 8]])
    descs = O.topology(ext, [5, 5, 4, 4, 4, 4], [1 / 16.0] * 3, 2)
    orc = O.Oracle(descs, 2)
    orc.coeff()
    ones = [np.ones((10, 10, 10)) for _ in descs]
    Ap = _apply_A(O, orc, ones, descs)
    assert max(np.abs(a).max() for a in Ap) == 0.0
    rng = np.random.default_rng(5)
    u = [rng.standard_normal((10, 10, 10)) for _ in descs]
    v = [rng.standard_normal((10, 10, 10)) for _ in descs]
    Au = _apply_A(O, orc, u, descs)
    Av = _apply_A(O, orc, v, descs)
    lhs = sum(float((a * b[1:-1, 1:-1, 1:-1]).sum()) for a, b in zip(Au, v))
    rhs = sum(float((a * b[1:-1, 1:-1, 1:-1]).sum()) for a, b in zip(Av, u))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_restriction_of_constant(oracle_mod):
    O = oracle_mod
    descs, orc = _one_block(O, (8, 8, 8), 2)
    orc.coeff()
    orc.put_phi(1, 0, np.zeros((10, 10, 10)))
    orc.put_rhs(1, 0, np.full((8, 8, 8), 0.75))
    orc.mgrestr(2)
    assert np.all(orc.get_rhs(2, 0) == 0.75)
    assert np.all(orc.get_phi(2, 0) == 0.0)


def test_prolongation_reproduces_linear(oracle_mod):
    O = oracle_mod
    ext = np.array([[0, 16, 0, 16, 0, 16]])
    descs = O.topology(ext, [5] * 6, [1 / 16.0] * 3, 2)  # periodic: no mgbound clamping
    orc = O.Oracle(descs, 2)
    orc.coeff()
    xc = np.arange(10) - 0.5  # coarse cell centres incl. ghosts, in coarse units
    lin = lambda X, Y, Z: 1.0 + 0.5 * X - 0.25 * Y + 0.125 * Z  # noqa: E731
    C = lin(xc[None, None, :], xc[None, :, None], xc[:, None, None])
    orc.put_phi(2, 0, C)
    orc.put_phi(1, 0, np.zeros((18, 18, 18)))
    orc.mgcorr(1)
    xf = (np.arange(18) - 0.5) / 2.0  # fine centres in coarse units
    F = lin(xf[None, None, :], xf[None, :, None], xf[:, None, None])
    np.testing.assert_allclose(orc.get_phi(1, 0), F, rtol=0, atol=1e-13)


@pytest.mark.parametrize("itrsch", [1, 2, 3])
def test_all_smoothers_converge(oracle_mod, itrsch):
    O = oracle_mod
    n = (16, 16, 16)
    descs, orc = _one_block(O, n, 3, itrsch=itrsch)
    orc.coeff()
    rng = np.random.default_rng(itrsch)
    b = rng.standard_normal(n)
    b -= b.mean()
    res = orc.solve([np.zeros((18, 18, 18))], [b], tol=1e-8, maxcy=200)
    assert res["status"] == 0
    h = res["history"]
    assert h[-1] <= 1e-8 and np.all(np.diff(np.log(h[: min(6, len(h))])) < 0)


def test_vcycle_factor_reasonable(oracle_mod):
    O = oracle_mod
    descs, orc = _one_block(O, (32, 32, 32), 5)
    orc.coeff()
    rng = np.random.default_rng(9)
    b = rng.standard_normal((32, 32, 32))
    b -= b.mean()
    res = orc.solve([np.zeros((34, 34, 34))], [b], tol=1e-9, maxcy=100)
    f = res["history"][1:4] / res["history"][0:3]
    assert np.all(f < 0.35)


def test_topology_matches_product(oracle_mod, h3d):
    O = oracle_mod
    from hydro3d_b200 import topology
    rng = np.random.default_rng(3)
    for trial in range(6):
        nb = rng.integers(1, 4, 3)
        bc = [5, 5, 4, 4, 4, 4] if trial % 2 else [4, 5, 5, 4, 5, 4][:6]
        bc = [bc[0], bc[0], bc[2], bc[2], bc[4], bc[4]]
        ext = []
        for k in range(nb[2]):
            for j in range(nb[1]):
                for i in range(nb[0]):
                    ext.append((4 * i, 4 * i + 4, 4 * j, 4 * j + 4, 4 * k, 4 * k + 4))
        ext = np.array(ext)
        od = O.topology(ext, bc, [0.1] * 3, 2)
        pd = topology.from_extents(ext, bc, [0.1] * 3, 2)
        for a, b in zip(od, pd):
            for f in ("nb_face", "nb_corner", "nb_edge", "nb_periodic", "bc", "n", "origin"):
                assert list(getattr(a, f)) == list(getattr(b, f)), (trial, f)
