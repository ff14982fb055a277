"""h3d_residual_noalloc (allocation-free residual norms) against h3d_mg_residual.

Both are called through the C ABI on the same fields; the allocation-free
entry point is called twice in a row on the same arrays and must give the
same answer both times.  The two sum in different orders, so the norms are
compared with a relative tolerance of 1e-12.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, P = 4, 5
RTOL = 1e-12


def _call(lib, p_dev, b_dev, n, h, phys, stream=None):
    import torch
    out = (C.c_double * 4)()
    hh = (C.c_double * 3)(*h)
    st = C.c_void_p(stream.cuda_stream) if stream is not None else None
    rc = lib.h3d_residual_noalloc(C.c_void_p(p_dev.data_ptr()), C.c_void_p(b_dev.data_ptr()),
                                  n[0], n[1], n[2], hh, phys, out, st)
    assert rc == 0, lib.h3d_mg_last_error(None)
    torch.cuda.synchronize()
    return np.array(out[:])


def _numpy_residual(p, b, n, h, phys):
    nx, ny, nz = n
    ax, ay, az = (1.0 / (x * x) for x in h)
    c = p[1:-1, 1:-1, 1:-1]
    acc = np.zeros_like(c)
    for (sl, a, bit) in (((slice(1, -1), slice(1, -1), slice(0, -2)), ax, 1),
                         ((slice(1, -1), slice(1, -1), slice(2, None)), ax, 2),
                         ((slice(1, -1), slice(0, -2), slice(1, -1)), ay, 4),
                         ((slice(1, -1), slice(2, None), slice(1, -1)), ay, 8),
                         ((slice(0, -2), slice(1, -1), slice(1, -1)), az, 16),
                         ((slice(2, None), slice(1, -1), slice(1, -1)), az, 32)):
        coef = np.full(c.shape, a)
        if phys & bit:
            edge = {1: (..., 0), 2: (..., -1), 4: (slice(None), 0), 8: (slice(None), -1),
                    16: (0,), 32: (-1,)}[bit]
            coef[edge] = 0.0
        acc += coef * (p[sl] - c)
    return b[1:-1, 1:-1, 1:-1] - acc


@pytest.mark.parametrize("bc,phys", [([W] * 6, 63), ([P, P, W, W, W, W], 60)])
def test_noalloc_matches_solver_residual(h3d, bc, phys):
    import torch
    n = (40, 24, 32)
    h = (0.025, 0.04, 0.03)
    blocks = h3d.topology.block_grid((1, 1, 1), n, bc, list(h), 3)
    rng = np.random.default_rng(77)
    shape = (n[2] + 2, n[1] + 2, n[0] + 2)
    p = rng.standard_normal(shape)
    b = np.zeros(shape)
    b[1:-1, 1:-1, 1:-1] = rng.standard_normal((n[2], n[1], n[0]))
    if not phys & 1:  # periodic x: ghosts hold the opposite interior plane
        p[:, :, 0] = p[:, :, n[0]]
        p[:, :, n[0] + 1] = p[:, :, 1]

    s = h3d.MultigridSolver(blocks, 3)
    s.upload("p", 0, p)
    s.upload("b", 0, b)
    rr, bb, rinf = s.residual()
    s.close()

    lib = h3d.lib()
    p_dev = torch.from_numpy(p).cuda()
    b_dev = torch.from_numpy(b).cuda()
    first = _call(lib, p_dev, b_dev, n, h, phys)
    second = _call(lib, p_dev, b_dev, n, h, phys)
    assert np.array_equal(first, second)
    for got, want in ((first[0], rr), (first[1], bb), (first[2], rinf)):
        assert abs(got - want) <= RTOL * abs(want), (got, want)
    r = _numpy_residual(p, b, n, h, phys)
    assert abs(first[3] - r.sum()) <= 1e-10 * np.abs(r).sum()
    assert np.array_equal(p_dev.cpu().numpy(), p) and np.array_equal(b_dev.cpu().numpy(), b)


def test_noalloc_rejects_oversize(h3d):
    import torch
    lib = h3d.lib()
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = (C.c_double * 4)()
    hh = (C.c_double * 3)(1.0, 1.0, 1.0)
    rc = lib.h3d_residual_noalloc(C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()),
                                  8, 257, 256, hh, 63, out, None)
    assert rc == h3d._lib.H3D_ERR_ARG
    assert b"65536" in lib.h3d_mg_last_error(None)


def test_noalloc_at_row_limit_on_a_stream(h3d):
    """ny*nz = 65536 rows exactly: the final quadruple lands in the last four
    doubles of the fixed device array.  Called on a caller-owned stream, twice,
    against a numpy evaluation of r = b - A p."""
    import torch
    n = (4, 256, 256)
    h = (0.5, 0.25, 0.125)
    phys = 63
    rng = np.random.default_rng(91)
    shape = (n[2] + 2, n[1] + 2, n[0] + 2)
    p = rng.standard_normal(shape)
    b = rng.standard_normal(shape)
    lib = h3d.lib()
    p_dev = torch.from_numpy(p).cuda()
    b_dev = torch.from_numpy(b).cuda()
    st = torch.cuda.Stream()
    first = _call(lib, p_dev, b_dev, n, h, phys, stream=st)
    second = _call(lib, p_dev, b_dev, n, h, phys, stream=st)
    assert np.array_equal(first, second)
    r = _numpy_residual(p, b, n, h, phys)
    bi = b[1:-1, 1:-1, 1:-1]
    assert abs(first[0] - (r * r).sum()) <= 1e-12 * (r * r).sum()
    assert abs(first[1] - (bi * bi).sum()) <= 1e-12 * (bi * bi).sum()
    assert abs(first[2] - np.abs(r).max() * h[0] * h[1] * h[2]) <= 1e-12 * np.abs(r).max()
    assert abs(first[3] - r.sum()) <= 1e-10 * np.abs(r).sum()


def test_noalloc_reports_nan(h3d):
    """A NaN in b shows in every entry of the result, max|r|*dV included."""
    import torch
    n = (16, 8, 8)
    rng = np.random.default_rng(5)
    shape = (n[2] + 2, n[1] + 2, n[0] + 2)
    p = rng.standard_normal(shape)
    b = rng.standard_normal(shape)
    b[4, 3, 7] = np.nan
    lib = h3d.lib()
    out = _call(lib, torch.from_numpy(p).cuda(), torch.from_numpy(b).cuda(), n, (1.0, 1.0, 1.0), 63)
    assert np.all(np.isnan(out)), out


def test_noalloc_refuses_a_capturing_stream(h3d):
    """The call copies its result to host memory and synchronises its stream,
    which a stream under graph capture does not allow: it must return
    H3D_ERR_ARG at once, before any work, and leave the capture intact."""
    import torch
    n = (8, 8, 8)
    lib = h3d._lib.lib()
    p = torch.zeros((n[2] + 2, n[1] + 2, n[0] + 2), dtype=torch.float64, device="cuda")
    b = torch.zeros_like(p)
    _call(lib, p, b, n, (0.1, 0.1, 0.1), 63)  # first call on the device: set-up outside any capture
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    out = (C.c_double * 4)()
    hh = (C.c_double * 3)(0.1, 0.1, 0.1)
    with torch.cuda.graph(g, stream=s):
        rc = lib.h3d_residual_noalloc(C.c_void_p(p.data_ptr()), C.c_void_p(b.data_ptr()), n[0], n[1], n[2], hh, 63,
                                      out, C.c_void_p(s.cuda_stream))
        p.add_(1.0)  # the capture itself stays valid
    assert rc == h3d._lib.H3D_ERR_ARG
    assert b"captured" in lib.h3d_mg_last_error(None)
    g.replay()
    torch.cuda.synchronize()
    assert float(p[1, 1, 1]) == 1.0
    del g
