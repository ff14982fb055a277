"""CPU: the C-ABI library loads and exports every entry point of include/h3d_mg.h."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "h3d_mg.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(h3d_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(h3d):
    L = h3d.lib()
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header(h3d):
    from hydro3d_b200 import _lib
    assert sorted(_lib.EXPORTS) == _declared()


def test_strerror_and_create_errors(h3d):
    import ctypes as C
    from hydro3d_b200 import _lib
    L = h3d.lib()
    assert L.h3d_mg_strerror(_lib.H3D_ERR_NOT_CONVERGED) == b"not converged"
    # a bad descriptor is rejected on the host before any device work
    blocks = h3d.topology.block_grid((1, 1, 1), (12, 12, 12), [4] * 6, [0.1] * 3, 4)
    d = _lib.MGDesc()
    arr = (_lib.BlockDesc * 1)(*blocks)
    d.nblocks, d.ngrd_gl, d.mg_itrsch, d.irestr, d.iproln, d.blocks = 1, 4, 3, 2, 1, arr
    h = C.c_void_p()
    assert L.h3d_mg_create(C.byref(h), C.byref(d)) == _lib.H3D_ERR_BAD_CONFIG  # 12 % 8 != 0
    assert b"divisible" in L.h3d_mg_last_error(None)
    d.ngrd_gl = 2
    for b in arr:
        b.ngrid = 2
    d.mg_itrsch = 4  # smoothers are 1 (GS-lex), 2 (line TDMA) and 3 (red-black GS)
    assert L.h3d_mg_create(C.byref(h), C.byref(d)) == _lib.H3D_ERR_BAD_CONFIG
    assert b"mg_itrsch" in L.h3d_mg_last_error(None)
    d.mg_itrsch = 3
    d.omega = 2.5  # over-relaxation of the FP32 sweeps: 0 (Gauss-Seidel) or in (0, 2)
    assert L.h3d_mg_create(C.byref(h), C.byref(d)) == _lib.H3D_ERR_BAD_CONFIG
    assert b"omega" in L.h3d_mg_last_error(None)
    d.omega = 1.25
    d.rb_order = 2  # 0: the reference's per-block order, 1: across block faces
    assert L.h3d_mg_create(C.byref(h), C.byref(d)) == _lib.H3D_ERR_BAD_CONFIG
    assert b"rb_order" in L.h3d_mg_last_error(None)


def test_product_does_not_touch_oracle():
    # the product package must not import, link or load the oracle
    for dp, _, fs in os.walk(os.path.join(ROOT, "hydro3d_b200")):
        for f in fs:
            if f.endswith((".py", ".cu", ".cpp", ".h", ".cuh")):
                txt = open(os.path.join(dp, f)).read()
                assert "oracle" not in txt.replace("oracle/", ""), f


def test_library_resolves_its_own_symbols():
    """Every symbol of the library's own namespace is defined in it (a
    launcher left inside an unnamed namespace would only fail at load time
    on the GPU machine)."""
    import subprocess
    out = subprocess.run(["nm", "-DC", os.path.join(ROOT, "hydro3d_b200", "libh3dmg.so")], capture_output=True,
                         text=True, check=True).stdout
    undef = [ln for ln in out.splitlines() if " U " in ln and ("h3d" in ln or "launch_" in ln)]
    assert not undef, undef
