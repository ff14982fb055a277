"""The mixed solver's coarsest level solved directly (coarse_direct): the
pseudo-inverse of the level's operator, applied inside the coarse cluster,
replaces its FP64 sweeps.  It must act like a converged sweep solve: the
same convergence as hundreds of coarsest sweeps, and the FP64 solution."""
import numpy as np
import pytest

from tests.helpers import interior_of_host, mean_removed_rel, to_oracle_descs

pytestmark = pytest.mark.gpu
W, P = 4, 5


def _problem(h3d, blocks, seed):
    rng = np.random.default_rng(seed)
    b, p = [], []
    for d in blocks:
        x = h3d.host_field(d)
        h3d.interior(x, d)[...] = rng.standard_normal((d.n[2], d.n[1], d.n[0]))
        b.append(x)
        p.append(h3d.host_field(d))
    m = np.mean(np.concatenate([h3d.interior(x, d).ravel() for x, d in zip(b, blocks)]))
    for x, d in zip(b, blocks):
        h3d.interior(x, d)[...] -= m
    return b, p


@pytest.mark.parametrize("layout", [((2, 2, 2), (16, 16, 16), [W] * 6, 4),
                                    ((2, 1, 2), (16, 16, 16), [P] * 6, 4),
                                    ((4, 2, 2), (32, 32, 32), [W] * 6, 5)])
def test_direct_coarsest_matches_converged_sweeps(h3d, oracle_mod, layout):
    nblk, n, bc, ngrid = layout
    blocks = h3d.topology.block_grid(nblk, n, bc, [1.0 / 32] * 3, ngrid, pl=1)
    b, _ = _problem(h3d, blocks, 41)
    hist = {}
    sol = {}
    for direct, csw in ((True, 32), (False, 400)):
        s = h3d.MultigridSolver(blocks, ngrid, precision="mixed", coarse_sweeps=csw, coarse_direct=direct)
        p = [h3d.host_field(d) for d in blocks]
        info = s.newsolv_mg(p, b, tol=1e-10, maxcy=100, history=True)
        assert info["converged"], (direct, info)
        hist[direct] = np.asarray(info["history"])
        sol[direct] = [interior_of_host(x, d) for x, d in zip(p, blocks)]
        s.close()
    # the same outer iterations, residuals within FP32 rounding of each other
    assert len(hist[True]) == len(hist[False])
    np.testing.assert_allclose(hist[True], hist[False], rtol=1e-2, atol=1e-12)
    orc = oracle_mod.Oracle(to_oracle_descs(oracle_mod, blocks), ngrid)
    orc.coeff()
    ref = orc.solve([np.zeros((d.n[2] + 2, d.n[1] + 2, d.n[0] + 2)) for d in blocks],
                    [interior_of_host(x, d) for x, d in zip(b, blocks)], tol=1e-12, maxcy=400)
    want = [x[1:-1, 1:-1, 1:-1] for x in ref["p"]]
    assert mean_removed_rel(sol[True], want) <= 1e-8


def test_direct_coarsest_is_fewer_launch_cycles_than_sweeps(h3d):
    """With coarse_direct the coarsest level takes no sweeps: the solve of a
    7-level configuration-3-like hierarchy (16 blocks of 64^3) needs no more
    V-cycles than with 32 sweeps and runs faster on the device."""
    blocks = h3d.topology.block_grid((4, 2, 2), (64, 64, 64), [W] * 6, [1.0 / 128] * 3, 6, pl=1)
    b, _ = _problem(h3d, blocks, 43)
    res = {}
    for direct in (False, True):
        s = h3d.MultigridSolver(blocks, 6, precision="mixed", coarse_sweeps=32, coarse_direct=direct)
        p = [h3d.host_field(d) for d in blocks]
        s.newsolv_mg([x.copy() for x in p], b, tol=1e-8, maxcy=100)  # warm-up, graphs captured
        for ib, d in enumerate(blocks):
            s.upload("b", ib, b[ib])
        s.zero_field("p")
        best = None
        for _ in range(3):
            s.zero_field("p")
            info = s.solve_resident(tol=1e-8, maxcy=100)
            best = info if best is None or info["device_ms"] < best["device_ms"] else best
        res[direct] = best
        s.close()
    assert res[True]["converged"] and res[False]["converged"]
    assert res[True]["cycles"] <= res[False]["cycles"]
    assert res[True]["device_ms"] < res[False]["device_ms"], (res[True]["device_ms"], res[False]["device_ms"])
