"""Failure detection of the solve (newsolv_mg.for:61-75), made on the host.

The reference prints 'not converged!!' when maxcy is reached and 'BIG RMAX'
and stops when the residual blows up; the library returns
H3D_ERR_NOT_CONVERGED and H3D_ERR_DIVERGED instead and the handle stays
usable.  No case here faults, traps or hangs the GPU: the failures come from
the inputs (a NaN in b, a cycle cap too small for the tolerance).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, P = 4, 5


def _problem(h3d, seed=3):
    blocks = h3d.topology.block_grid((2, 1, 1), (16, 16, 16), [P, P, W, W, W, W], [1.0 / 32] * 3, 3)
    rng = np.random.default_rng(seed)
    b, p = [], []
    for d in blocks:
        x = h3d.host_field(d)
        h3d.interior(x, d)[...] = rng.standard_normal((d.n[2], d.n[1], d.n[0]))
        b.append(x)
        p.append(h3d.host_field(d))
    m = np.mean([h3d.interior(x, d).mean() for x, d in zip(b, blocks)])
    for x, d in zip(b, blocks):
        h3d.interior(x, d)[...] -= m
    return blocks, b, p


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cycle_cap_reports_not_converged(h3d, precision):
    blocks, b, p = _problem(h3d)
    s = h3d.MultigridSolver(blocks, 3, precision=precision)
    info = s.newsolv_mg([x.copy() for x in p], b, tol=1e-12, maxcy=1)
    assert not info["converged"]
    assert info["status"] == h3d._lib.H3D_ERR_NOT_CONVERGED
    assert info["outer"] == 1 and info["relres"] > 1e-12
    # the handle stays usable: the same solve with a budget converges
    info = s.newsolv_mg([x.copy() for x in p], b, tol=1e-8, maxcy=200)
    assert info["converged"] and info["relres"] <= 1e-8
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nan_in_rhs_reports_diverged(h3d, precision):
    blocks, b, p = _problem(h3d)
    bad = [x.copy() for x in b]
    d = blocks[1]
    bad[1][d.pl + 3, d.pl + 5, d.pl + 7] = np.nan
    s = h3d.MultigridSolver(blocks, 3, precision=precision)
    with pytest.raises(h3d.H3DError) as e:
        s.newsolv_mg([x.copy() for x in p], bad, tol=1e-8, maxcy=50)
    assert e.value.code == h3d._lib.H3D_ERR_DIVERGED
    info = s.newsolv_mg([x.copy() for x in p], b, tol=1e-8, maxcy=200)
    assert info["converged"]
    s.close()


def test_incompatible_rhs_reports_not_converged(h3d):
    """A right-hand side with a mean on a problem without Dirichlet faces is
    not in the range of the operator: the residual stagnates at its mean
    part and the solve ends at maxcy as not converged."""
    blocks, b, p = _problem(h3d)
    s = h3d.MultigridSolver(blocks, 3)
    off = [x.copy() for x in b]
    for x, d in zip(off, blocks):
        h3d.interior(x, d)[...] += 1.0  # incompatible with the Neumann operator
    info = s.newsolv_mg([x.copy() for x in p], off, tol=1e-8, maxcy=20)
    assert info["status"] == h3d._lib.H3D_ERR_NOT_CONVERGED
    s.close()


def test_bounded_device_wait_reports_timeout(h3d):
    """A device wait on an mbarrier that nothing arrives at (the sweeps' own
    bounded-wait routine) gives up after the limit set at run time (2^20
    clocks, about half a millisecond), the host reads H3D_ERR_TIMEOUT, and
    the same handle then solves the problem.  No copy is in flight and
    nothing faults: the wait simply runs out."""
    import time
    blocks, b, p = _problem(h3d)
    s = h3d.MultigridSolver(blocks, 3, use_graph=False)
    s.coeff()
    s.set_wait_limit(1 << 20)
    try:
        t0 = time.perf_counter()
        assert s.wait_probe() == h3d._lib.H3D_ERR_TIMEOUT
        assert time.perf_counter() - t0 < 5.0
        # a solve under the short limit still completes (its copies land in microseconds)
        info = s.newsolv_mg([x.copy() for x in p], b, tol=1e-8, maxcy=200)
        assert info["converged"]
    finally:
        s.set_wait_limit(0)
    assert s.wait_probe() == h3d._lib.H3D_ERR_TIMEOUT  # the default limit runs out too (tens of ms)
    info = s.newsolv_mg([x.copy() for x in p], b, tol=1e-8, maxcy=200)
    assert info["converged"] and info["relres"] <= 1e-8
    s.close()
