"""GPU parity at the benchmark configurations' own sizes, through the C ABI.

Every case builds the workload with the seeded generators (hydro3d_b200.synth)
and runs the CUDA path against the oracle on the same inputs:

  config 1  64^3 single block, full FP64 solve to 1e-8: cycle count equal to
            the oracle's, residual history within 1e-9, pressure (mean
            removed) within 1e-7.
  config 2  192^3 as 2x2x2 blocks of 96^3, periodic x, warm start from the
            converged pressure of the seed-1017 problem: as config 1.
  config 3  512x256x256 as 4x2x2 blocks of 128^3, 7 levels: two V-cycles on
            the level state bit for bit, then two outer FP64 iterations
            (history within 1e-12, iterate within 1e-12).
  config 4  27 uneven independent blocks: one V-cycle bit for bit on every
            block; the mixed-precision solve reaches 1e-8 in every block.
  config 5  256^3, 1000:1 density (L_LSM coefficients): two V-cycles bit for
            bit.
"""
import numpy as np
import pytest

from tests.helpers import interior_of_host, mean_removed_rel, to_oracle_descs

pytestmark = pytest.mark.gpu

THREADS = 16


def _oracle(O, prob):
    orc = O.Oracle(to_oracle_descs(O, prob.blocks), prob.ngrid, 3, 2, 1, lsm=prob.var_coef, threads=THREADS)
    if prob.var_coef:
        for ib, (d, x) in enumerate(zip(prob.blocks, prob.dens)):
            orc.set_density(ib, interior_of_host(x, d))
    orc.coeff()
    return orc


def _solver(h3d, prob, precision="fp64", **kw):
    s = h3d.MultigridSolver(prob.blocks, prob.ngrid, precision=precision, var_coef=prob.var_coef, maxcy=400, **kw)
    if prob.var_coef:
        for ib, d in enumerate(prob.dens):
            s.set_density(ib, d)
    s.coeff()
    return s


def _canon(x, d):
    p = d.pl
    return np.ascontiguousarray(x[p - 1:p + d.n[2] + 1, p - 1:p + d.n[1] + 1, p - 1:p + d.n[0] + 1])


def _oracle_solve(orc, prob, tol=1e-8, maxcy=400):
    return orc.solve([_canon(x, d) for x, d in zip(prob.p0, prob.blocks)],
                     [interior_of_host(x, d) for x, d in zip(prob.b, prob.blocks)], tol=tol, maxcy=maxcy)


def _gpu_solve(s, prob, tol=1e-8, maxcy=400):
    p = [x.copy() for x in prob.p0]
    info = s.newsolv_mg(p, prob.b, tol=tol, maxcy=maxcy, history=True)
    return p, info


def _compare_solves(h3d, O, prob):
    orc = _oracle(O, prob)
    ref = _oracle_solve(orc, prob)
    orc.close()
    s = _solver(h3d, prob)
    p, info = _gpu_solve(s, prob)
    s.close()
    assert ref["status"] == 0 and info["converged"]
    assert info["cycles"] == ref["cycles"], (info["cycles"], ref["cycles"])
    np.testing.assert_allclose(info["history"], ref["history"], rtol=1e-9, atol=0)
    got = [interior_of_host(x, d) for x, d in zip(p, prob.blocks)]
    want = [x[1:-1, 1:-1, 1:-1] for x in ref["p"]]
    assert mean_removed_rel(got, want) <= 1e-7


def test_config1_solve_matches_oracle(oracle_mod, h3d):
    from hydro3d_b200 import synth
    _compare_solves(h3d, oracle_mod, synth.config1())


def test_config2_warm_start_matches_oracle(oracle_mod, h3d):
    """The warm start is the oracle's converged pressure of the seed-1017
    problem, given to both solvers."""
    from hydro3d_b200 import host_field, interior, synth
    prev = synth.config2(seed=1017)
    orc = _oracle(oracle_mod, prev)
    r = _oracle_solve(orc, prev)
    orc.close()
    assert r["status"] == 0
    fields = [host_field(d) for d in prev.blocks]
    for x, d, pr in zip(fields, prev.blocks, r["p"]):
        interior(x, d)[...] = pr[1:-1, 1:-1, 1:-1]
    prob = synth.config2(p0=synth.gather(fields, prev.blocks))
    _compare_solves(h3d, oracle_mod, prob)


def _vcycles_bitexact(h3d, O, prob, ncycles=2, blocks=None):
    orc = _oracle(O, prob)
    s = _solver(h3d, prob)
    for ib, d in enumerate(prob.blocks):
        phi = _canon(prob.p0[ib], d)
        rhs = interior_of_host(prob.b[ib], d)
        s.put_level(1, "phi", ib, phi)
        s.put_level(1, "rhs", ib, rhs)
        orc.put_phi(1, ib, phi)
        orc.put_rhs(1, ib, rhs)
    for _ in range(ncycles):
        s.vcycle()
        orc.vcycle()
    for ib in (range(len(prob.blocks)) if blocks is None else blocks):
        a, b = s.get_level(1, "phi", ib), orc.get_phi(1, ib)
        assert np.array_equal(a, b), (ib, float(np.abs(a - b).max()))
    s.close()
    return orc


def test_config3_vcycles_bitexact_and_outer_steps(oracle_mod, h3d):
    from hydro3d_b200 import synth
    prob = synth.config3()
    orc = _vcycles_bitexact(h3d, oracle_mod, prob)
    ref = _oracle_solve(orc, prob, tol=1e-30, maxcy=2)
    orc.close()
    s = _solver(h3d, prob)
    p, info = _gpu_solve(s, prob, tol=1e-30, maxcy=2)
    s.close()
    assert info["cycles"] == ref["cycles"] == 2
    np.testing.assert_allclose(info["history"], ref["history"], rtol=1e-12, atol=0)
    got = [interior_of_host(x, d) for x, d in zip(p, prob.blocks)]
    want = [x[1:-1, 1:-1, 1:-1] for x in ref["p"]]
    assert mean_removed_rel(got, want) <= 1e-12


def test_config4_uneven_blocks(oracle_mod, h3d):
    """27 independent blocks of 15+ different shapes in one solver: one
    V-cycle bit for bit on every block, then the mixed-precision solve with
    the per-block stop rule (every block's ||r||/||b|| <= 1e-8, recomputed
    here by the oracle from the returned pressure), and every block's error
    against the oracle's solution to 1e-12 within the bound the residual
    sets: ||e|| <= ||r|| / lambda_min, lambda_min = (4/h^2) sin^2(pi/(2 n))
    the smallest non-zero eigenvalue of the block's Neumann operator (n its
    longest axis).  Long thin blocks make that bound large: a residual of
    1e-8 allows errors near 1e-4 there."""
    from hydro3d_b200 import synth
    prob = synth.config4()
    sizes = {tuple(d.n) for d in prob.blocks}
    assert len(sizes) > 10
    orc = _vcycles_bitexact(h3d, oracle_mod, prob, ncycles=1)
    ref = _oracle_solve(orc, prob, tol=1e-12, maxcy=600)
    assert ref["status"] == 0
    s = _solver(h3d, prob, precision="mixed")
    p = [x.copy() for x in prob.p0]
    info = s.newsolv_mg(p, prob.b, tol=1e-8, maxcy=400, stop_rule=2)
    s.close()
    assert info["converged"] and info["relres_block_max"] <= 1e-8
    r, _, _, _ = orc.residual([_canon(x, d) for x, d in zip(p, prob.blocks)],
                              [interior_of_host(x, d) for x, d in zip(prob.b, prob.blocks)])
    orc.close()
    for rb, x, d in zip(r, prob.b, prob.blocks):
        assert np.linalg.norm(rb) <= 1.0001e-8 * np.linalg.norm(interior_of_host(x, d))
    for rb, x, d, w in zip(r, p, prob.blocks, ref["p"]):
        g = interior_of_host(x, d)
        w = w[1:-1, 1:-1, 1:-1]
        e = (g - g.mean()) - (w - w.mean())
        hh = d.h[0]
        lam = 4.0 / (hh * hh) * np.sin(np.pi / (2 * max(d.n))) ** 2
        assert np.linalg.norm(e) <= 1.01 * np.linalg.norm(rb) / lam + 1e-12 * np.linalg.norm(w), tuple(d.n)


def test_config5_lsm_vcycles_bitexact(oracle_mod, h3d):
    from hydro3d_b200 import synth
    prob = synth.config5()
    orc = _vcycles_bitexact(h3d, oracle_mod, prob)
    orc.close()
