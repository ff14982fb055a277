"""Golden fixtures from the reference's own Fortran (tests/golden/*.npz).

tests/golden/make_golden.py ran the reference's coeff + mgkcyc, translated
statement by statement from mgsolver.for / exchangepp.for /
localparameters.for by oracle/fortran_ref.py, on seeded inputs.  Here:
  * the oracle reproduces every fixture bit for bit (this pins the oracle);
  * the CUDA path (FP64, through the C ABI) reproduces every fixture bit for
    bit, with the fixture's own smoother (red-black GS, lexicographic GS or
    line TDMA);
  * where the reference source tree is present (not on GPU machines), the
    fixtures are regenerated and must be identical (the generator is
    deterministic).
"""
import glob
import os

import numpy as np
import pytest

from tests.helpers import to_oracle_descs

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(glob.glob(os.path.join(GOLDEN, "mgkcyc_*.npz")))
NAMES = [os.path.basename(f)[len("mgkcyc_"):-len(".npz")] for f in FILES]


def _load(name):
    with np.load(os.path.join(GOLDEN, "mgkcyc_%s.npz" % name)) as z:
        return {k: z[k] for k in z.files}


def test_fixtures_present():
    assert len(NAMES) >= 12
    assert sum(n.startswith("lmr_") for n in NAMES) >= 5


def _layout(g, topo):
    """Descriptors of a fixture's layout: topo(ext, bc, h, ngrid) builds the
    unrefined blocks; LMR fixtures then refine them by their rdiv."""
    ngrd = int(g["ngrd_gl"])
    if "rdiv" not in g:
        return list(topo(g["ext"], g["bc"], g["h"], ngrd))
    from hydro3d_b200.topology import refine
    rdiv = [int(r) for r in g["rdiv"]]
    ngi = ngrd - (max(rdiv).bit_length() - 1)
    return refine(list(topo(g["ext"], g["bc"], g["h"], ngi)), rdiv, ngi)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference(oracle_mod, name):
    g = _load(name)
    O = oracle_mod
    descs = _layout(g, O.topology)
    nb = int(g["nblocks"])
    orc = O.Oracle(list(descs), int(g["ngrd_gl"]), int(g["mg_itrsch"]), 2, 1, lsm=bool(g["lsm"]))
    if g["lsm"]:
        for ib in range(nb):
            orc.set_density(ib, g["dens_%d" % ib])
    orc.coeff()
    out = orc.mgkcyc([g["pp_in_%d" % ib] for ib in range(nb)], [g["su_%d" % ib] for ib in range(nb)])
    for ib in range(nb):
        ref = g["pp_out_%d" % ib]
        assert np.array_equal(out[ib], ref), (name, ib, float(np.abs(out[ib] - ref).max()))
    orc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_matches_reference(h3d, name):
    g = _load(name)
    nb = int(g["nblocks"])
    ngrd = int(g["ngrd_gl"])
    blocks = _layout(g, lambda e, b, h, n: h3d.topology.from_extents(e, b, h, n, pl=1))
    s = h3d.MultigridSolver(blocks, ngrd, mg_itrsch=int(g["mg_itrsch"]), var_coef=bool(g["lsm"]))
    if g["lsm"]:
        for ib, d in enumerate(blocks):
            dens = h3d.host_field(d)
            h3d.interior(dens, d)[...] = g["dens_%d" % ib]
            s.set_density(ib, dens)
        s.coeff()
    pp = [np.ascontiguousarray(g["pp_in_%d" % ib]) for ib in range(nb)]
    su = []
    for ib, d in enumerate(blocks):
        a = h3d.host_field(d)
        h3d.interior(a, d)[...] = g["su_%d" % ib]
        su.append(a)
    s.mgkcyc(pp, su)
    for ib in range(nb):
        ref = g["pp_out_%d" % ib]
        assert np.array_equal(pp[ib], ref), (name, ib, float(np.abs(pp[ib] - ref).max()))
    s.close()


def _make_golden():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


def _reference_tree():
    src = _make_golden().REF_SRC
    return src if os.path.isfile(os.path.join(src, "mgsolver.for")) else None


@pytest.mark.skipif(_reference_tree() is None, reason="reference source tree not present")
@pytest.mark.parametrize("name", ["walls_2x1x1", "lsm_periodic_x_2x1x2", "periodic_x_2x2x2", "lmr_corners_2x2x2"])
def test_fixture_regenerates(oracle_mod, name):
    fresh = _make_golden().run_case(name)
    old = _load(name)
    assert sorted(fresh) == sorted(old)
    for k in old:
        assert np.array_equal(np.asarray(fresh[k]), old[k]), k


# -- the projection: calvel, calmas, exchange(1..4), pbound in newsolv_mg's loop
PFILES = sorted(glob.glob(os.path.join(GOLDEN, "project_*.npz")))
PNAMES = [os.path.basename(f)[len("project_"):-len(".npz")] for f in PFILES]


def _pload(name):
    with np.load(os.path.join(GOLDEN, "project_%s.npz" % name)) as z:
        return {k: z[k] for k in z.files}


def _face_mask(shape):
    """Interior cells and face ghosts: what the projection defines (the
    reference's exchanges also write edge and corner ghosts, which neither
    calvel nor calmas reads)."""
    g = [(np.arange(n) == 0) | (np.arange(n) == n - 1) for n in shape]
    return (g[0][:, None, None].astype(int) + g[1][None, :, None] + g[2][None, None, :]) <= 1


def test_projection_fixtures_present():
    assert len(PNAMES) >= 4


@pytest.mark.parametrize("name", PNAMES)
def test_oracle_projection_matches_reference(oracle_mod, name):
    g = _pload(name)
    O = oracle_mod
    nb, lsm = int(g["nblocks"]), bool(g["lsm"])
    descs = O.topology(g["ext"], g["bc"], g["h"], int(g["ngrd_gl"]))
    orc = O.Oracle(list(descs), int(g["ngrd_gl"]), 3, 2, 1, lsm=lsm)
    dens = [g["dens_%d" % ib] for ib in range(nb)] if lsm else None
    if lsm:
        for ib in range(nb):
            orc.set_density(ib, dens[ib][1:-1, 1:-1, 1:-1])
    orc.coeff()
    f = {k: [g["%s_in_%d" % (k, ib)] for ib in range(nb)] for k in ("p", "u", "v", "w", "ustar", "vstar", "wstar")}
    res = orc.project(f["p"], f["u"], f["v"], f["w"], f["ustar"], f["vstar"], f["wstar"], float(g["dt"]),
                      float(g["alfapr"]), dens=dens, tol=0.0, maxcy=int(g["niter"]), stop_rule=1)
    assert res["cycles"] == int(g["niter"])
    assert np.array_equal(res["history"], g["rmax"]), (res["history"], g["rmax"])
    su, _, _ = orc.calmas(res["u"], res["v"], res["w"], float(g["dt"]))
    for ib in range(nb):
        m = _face_mask(res["p"][ib].shape)
        for k in ("p", "u", "v", "w"):
            got, want = res[k][ib], g["%s_out_%d" % (k, ib)]
            assert np.array_equal(got[m], want[m]), (name, k, ib, float(np.abs(got[m] - want[m]).max()))
        assert np.array_equal(su[ib], g["su_out_%d" % ib])
    orc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", PNAMES)
def test_cuda_projection_matches_reference(h3d, name):
    g = _pload(name)
    nb, lsm = int(g["nblocks"]), bool(g["lsm"])
    ngrd = int(g["ngrd_gl"])
    blocks = h3d.topology.from_extents(g["ext"], g["bc"], g["h"], ngrd, pl=1)
    s = h3d.MultigridSolver(blocks, ngrd, var_coef=lsm)
    if lsm:
        for ib in range(nb):
            s.set_density(ib, np.ascontiguousarray(g["dens_%d" % ib]))
    s.coeff()
    f = {k: [np.ascontiguousarray(g["%s_in_%d" % (k, ib)]) for ib in range(nb)]
         for k in ("p", "u", "v", "w", "ustar", "vstar", "wstar")}
    info = s.project(f["p"], f["u"], f["v"], f["w"], f["ustar"], f["vstar"], f["wstar"], float(g["dt"]),
                     float(g["alfapr"]), tol=0.0, maxcy=int(g["niter"]), stop_rule=1, history=True)
    assert info["outer"] == int(g["niter"]) and not info["converged"]
    assert np.array_equal(info["history"], g["rmax"])
    for ib, d in enumerate(blocks):
        m = _face_mask(f["p"][ib].shape)
        for k in ("p", "u", "v", "w"):
            got, want = f[k][ib], g["%s_out_%d" % (k, ib)]
            assert np.array_equal(got[m], want[m]), (name, k, ib, float(np.abs(got[m] - want[m]).max()))
        b = h3d.host_field(d)
        s.download("b", ib, b)
        assert np.array_equal(h3d.interior(b, d), g["su_out_%d" % ib])
    s.close()


@pytest.mark.skipif(_reference_tree() is None, reason="reference source tree not present")
@pytest.mark.parametrize("name", ["walls_2x1x1", "lsm_periodic_y_2x2x1"])
def test_projection_fixture_regenerates(oracle_mod, name):
    fresh = _make_golden().run_projection_case(name)
    old = _pload(name)
    assert sorted(fresh) == sorted(old)
    for k in old:
        assert np.array_equal(np.asarray(fresh[k]), old[k]), k


# -- the SIP pressure path (sipsol.for, pressure_1sweep's loop)
SFILES = sorted(glob.glob(os.path.join(GOLDEN, "sip_*.npz")))
SNAMES = [os.path.basename(f)[len("sip_"):-len(".npz")] for f in SFILES]


def _sload(name):
    with np.load(os.path.join(GOLDEN, "sip_%s.npz" % name)) as z:
        return {k: z[k] for k in z.files}


def test_sip_fixtures_present():
    assert len(SNAMES) >= 3


@pytest.mark.parametrize("name", SNAMES)
def test_oracle_sip_matches_reference(oracle_mod, name):
    g = _sload(name)
    O = oracle_mod
    nb = int(g["nblocks"])
    descs = O.topology(g["ext"], g["bc"], g["h"], 2)
    orc = O.Oracle(list(descs), 2, 3, 2, 1)
    orc.coeff()
    f = {k: [g["%s_in_%d" % (k, ib)] for ib in range(nb)] for k in ("p", "u", "v", "w", "ustar", "vstar", "wstar")}
    res = orc.pressure_1sweep(f["p"], f["u"], f["v"], f["w"], f["ustar"], f["vstar"], f["wstar"], float(g["dt"]),
                              float(g["alfapr"]), eps=0.0, niter=int(g["niter"]), nswp=int(g["nswp"]))
    assert res["iters"] == int(g["niter"])
    assert np.array_equal(res["history"], g["rmax"])
    assert res["nsweeps"] == int(np.sum(g["nsweep"]))
    for ib in range(nb):
        m = _face_mask(res["p"][ib].shape)
        for k in ("p", "u", "v", "w"):
            got, want = res[k][ib], g["%s_out_%d" % (k, ib)]
            assert np.array_equal(got[m], want[m]), (name, k, ib, float(np.abs(got[m] - want[m]).max()))
    orc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", SNAMES)
def test_cuda_sip_matches_reference(h3d, name):
    g = _sload(name)
    nb = int(g["nblocks"])
    blocks = h3d.topology.from_extents(g["ext"], g["bc"], g["h"], 2, pl=1)
    s = h3d.MultigridSolver(blocks, 2)
    for k in ("p", "u", "v", "w", "ustar", "vstar", "wstar"):
        for ib in range(nb):
            s.upload(k, ib, np.ascontiguousarray(g["%s_in_%d" % (k, ib)]))
    info = s.pressure_1sweep(float(g["dt"]), float(g["alfapr"]), eps=0.0, niter=int(g["niter"]),
                             nswp=int(g["nswp"]))
    assert info["outer"] == int(g["niter"]) and info["cycles"] == int(np.sum(g["nsweep"]))
    assert np.array_equal(info["history"], g["rmax"])
    for ib, d in enumerate(blocks):
        for k in ("p", "u", "v", "w"):
            host = h3d.host_field(d)
            s.download(k, ib, host)
            want = g["%s_out_%d" % (k, ib)]
            m = _face_mask(want.shape)
            assert np.array_equal(host[m], want[m]), (name, k, ib, float(np.abs(host[m] - want[m]).max()))
    s.close()


@pytest.mark.skipif(_reference_tree() is None, reason="reference source tree not present")
def test_sip_fixture_regenerates(oracle_mod):
    fresh = _make_golden().run_sip_case("periodic_x_2x2x1")
    old = _sload("periodic_x_2x2x1")
    assert sorted(fresh) == sorted(old)
    for k in old:
        assert np.array_equal(np.asarray(fresh[k]), old[k]), k
