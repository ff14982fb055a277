"""GPU parity of the SIP pressure path (sipsol.for:2-205, press.for:382-519)
through the C ABI against the oracle: the LU factors and both substitutions
are recurrences over neighbours, run on the device as hyperplane wavefronts
(one CTA per block); every value is the reference's, so the correction pp is
compared bit for bit.  The per-sweep sum |res| is added in another order
(per-thread partials), so it is compared to 1e-12 relative, and the sweep
count, which it decides, must be equal."""
import numpy as np
import pytest

from tests.helpers import projection_fields, to_host, to_oracle_descs

pytestmark = pytest.mark.gpu

W, P = 4, 5
LAYOUTS = [
    ((1, 1, 1), (16, 16, 16), [W] * 6),
    ((2, 2, 2), (8, 16, 8), [P, P, W, W, W, W]),
    ((2, 1, 3), (8, 8, 16), [P] * 6),
    ((3, 2, 1), (16, 8, 8), [W, W, P, P, W, W]),
]


def _pair(O, h3d, layout):
    nblk, n, bc = layout
    blocks = h3d.topology.block_grid(nblk, n, bc, [1.0 / 32] * 3, 2)
    s = h3d.MultigridSolver(blocks, 2)
    orc = O.Oracle(to_oracle_descs(O, blocks), 2, 3, 2, 1)
    orc.coeff()
    return blocks, s, orc


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("nswp", [3, 200])
def test_sipsol_bitexact(oracle_mod, h3d, layout, nswp):
    blocks, s, orc = _pair(oracle_mod, h3d, layout)
    rng = np.random.default_rng(21)
    pp = [rng.standard_normal((d.n[2] + 2, d.n[1] + 2, d.n[0] + 2)) for d in blocks]
    su = [rng.standard_normal((d.n[2], d.n[1], d.n[0])) for d in blocks]
    want, ns, hist = orc.sipsol(pp, su, nswp)
    for ib, d in enumerate(blocks):
        s.upload("pp", ib, to_host([d], [pp[ib]])[0])
        b = h3d.host_field(d)
        h3d.interior(b, d)[...] = su[ib]
        s.upload("b", ib, b)
    ns_gpu, resab = s.sipsol(nswp)
    assert ns_gpu == ns, (ns_gpu, ns)
    assert resab == pytest.approx(hist[-1], rel=1e-12)
    for ib, d in enumerate(blocks):
        host = h3d.host_field(d)
        s.download("pp", ib, host)
        got = np.ascontiguousarray(h3d.with_ghost(host, d))
        assert np.array_equal(got, want[ib]), (ib, float(np.abs(got - want[ib]).max()))
    s.close()


@pytest.mark.parametrize("layout", LAYOUTS[1:3])
def test_pressure_1sweep_matches_oracle(oracle_mod, h3d, layout):
    """The whole SIP pressure loop on the velocities, 4 iterations of at most
    30 sweeps: rmax after every calmas and p, u, v, w (interior and face
    ghosts) bit for bit."""
    blocks, s, orc = _pair(oracle_mod, h3d, layout)
    f = projection_fields(blocks, 31)
    ref = orc.pressure_1sweep(f["p"], f["u"], f["v"], f["w"], f["us"], f["vs"], f["ws"], 0.5, 1.0, eps=0.0,
                              niter=4, nswp=30)
    for k, name in (("p", "p"), ("u", "u"), ("v", "v"), ("w", "w"), ("us", "ustar"), ("vs", "vstar"),
                    ("ws", "wstar")):
        for ib, x in enumerate(to_host(blocks, f[k])):
            s.upload(name, ib, x)
    info = s.pressure_1sweep(0.5, 1.0, eps=0.0, niter=4, nswp=30)
    assert info["outer"] == ref["iters"] == 4 and info["cycles"] == ref["nsweeps"]
    np.testing.assert_array_equal(info["history"], ref["history"])
    for ib, d in enumerate(blocks):
        for k in ("p", "u", "v", "w"):
            host = h3d.host_field(d)
            s.download(k, ib, host)
            got = np.ascontiguousarray(h3d.with_ghost(host, d))
            g = [(np.arange(n) == 0) | (np.arange(n) == n - 1) for n in got.shape]
            m = (g[0][:, None, None].astype(int) + g[1][None, :, None] + g[2][None, None, :]) <= 1
            assert np.array_equal(got[m], ref[k][ib][m]), (k, ib)
    s.close()


def test_sip_rejects_variable_coefficients(h3d):
    blocks = h3d.topology.block_grid((1, 1, 1), (8, 8, 8), [W] * 6, [1.0 / 8] * 3, 2)
    s = h3d.MultigridSolver(blocks, 2, var_coef=True)
    with pytest.raises(h3d.H3DError) as e:
        s.sipsol(3)
    assert e.value.code == h3d._lib.H3D_ERR_BAD_CONFIG
    s.close()
