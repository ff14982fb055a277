"""CPU: the product's ghost-fill tables reproduce the reference's level exchange.

The library resolves mgbound + exchangepp + exchbc_mgpp on cell identities
(hydro3d_b200/csrc/h3d_halo.cpp); applying that gather to random level data
must give exactly what the oracle's value-by-value restatement of the same
Fortran routines gives.
"""
import numpy as np
import pytest

from tests.helpers import to_oracle_descs

W, P = 4, 5
CASES = [
    ((1, 1, 1), (8, 8, 8), [W] * 6, 2, 1),
    ((2, 2, 2), (8, 8, 8), [W] * 6, 2, 1),
    ((2, 2, 2), (8, 8, 8), [P, P, W, W, W, W], 2, 2),
    ((3, 2, 2), (8, 4, 8), [P, P, W, W, W, W], 3, 1),
    ((2, 3, 2), (8, 8, 8), [W, W, P, P, P, P], 3, 2),
    ((1, 1, 1), (8, 8, 8), [P] * 6, 2, 1),
    ((3, 3, 3), (4, 4, 4), [P] * 6, 2, 1),
    ((4, 1, 2), (4, 8, 4), [W, W, W, W, P, P], 2, 2),
]


def _ref_fill(O, blocks, g, kind, phis):
    orc = O.Oracle(to_oracle_descs(O, blocks), blocks[0].ngrid)
    orc.coeff()
    for ib, a in enumerate(phis):
        orc.put_phi(g, ib, a)
    if kind in (0, 3):
        orc.mgbound(g)
        orc.exchangepp(g)
    elif kind == 1:
        orc.exchangepp(g)
    else:
        orc.mgbound(g)
    return np.concatenate([orc.get_phi(g, ib).ravel() for ib in range(len(blocks))])


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_halo_table_matches_oracle(oracle_mod, h3d, case, kind):
    O = oracle_mod
    nblk, n, bc, ngrid, g = case
    blocks = h3d.topology.block_grid(nblk, n, bc, [1 / 16.0] * 3, ngrid)
    rng = np.random.default_rng(hash((nblk, n, g, kind)) % 2**32)
    phis = []
    for d in blocks:
        s = 2 ** (g - 1)
        phis.append(rng.standard_normal((d.n[2] // s + 2, d.n[1] // s + 2, d.n[0] // s + 2)))
    ref = _ref_fill(O, blocks, g, kind, phis)
    flat = np.concatenate([a.ravel() for a in phis])
    dst, src = h3d.halo_table(blocks, g, kind)
    out = flat.copy()
    out[dst] = flat[src & 0x7FFFFFFF]
    assert np.array_equal(out, ref)
    if kind == 0:
        # after a sweep every ghost resolves to a current interior value
        assert not np.any(src & 0x80000000)


def test_face_table_is_subset(h3d):
    blocks = h3d.topology.block_grid((2, 2, 1), (8, 8, 8), [P, P, W, W, W, W], [0.1] * 3, 2)
    d0, s0 = h3d.halo_table(blocks, 1, 0)
    d3, s3 = h3d.halo_table(blocks, 1, 3)
    m = dict(zip(d0.tolist(), s0.tolist()))
    assert len(d3) > 0 and all(m[a] == b for a, b in zip(d3.tolist(), s3.tolist()))


def test_uneven_face_neighbours_rejected(h3d):
    # a face neighbour must have identical extents (read_infodom only pairs equal faces)
    ext = np.array([[0, 8, 0, 8, 0, 8], [8, 16, 0, 4, 0, 8]])
    blocks = h3d.topology.from_extents(ext, [W] * 6, [0.1] * 3, 2)
    assert blocks[0].nb_face[1] == -1 and blocks[1].nb_face[0] == -1


@pytest.mark.parametrize("case", CASES)
def test_sweep_face_ghosts_are_pushable(h3d, case):
    """The register-window sweeps write whole ghost faces themselves (ghost
    pushes): a face qualifies when every one of its ghosts is filled from the
    adjacent interior face of one block, cell for cell.  On these regular
    layouts every face ghost does (walls from the block itself, neighbours and
    periodic partners from the facing block), so only edges and corners are
    left to the gather."""
    nblk, n, bc, ngrid, g = case
    blocks = h3d.topology.block_grid(nblk, n, bc, [1 / 16.0] * 3, ngrid)
    s = 2 ** (g - 1)
    dims = [(d.n[0] // s, d.n[1] // s, d.n[2] // s) for d in blocks]
    starts = np.cumsum([0] + [(x + 2) * (y + 2) * (z + 2) for x, y, z in dims])

    def locate(i):
        b = int(np.searchsorted(starts, i, side="right") - 1)
        nx, ny, _ = dims[b]
        l = i - starts[b]
        return b, l % (nx + 2), (l // (nx + 2)) % (ny + 2), l // ((nx + 2) * (ny + 2))

    dst, src = h3d.halo_table(blocks, g, 0)
    faces = {}
    for d, sv in zip(dst, src):
        b, x, y, z = locate(int(d))
        nx, ny, nz = dims[b]
        out = [x in (0, nx + 1), y in (0, ny + 1), z in (0, nz + 1)]
        if sum(out) != 1:
            continue
        axis = out.index(True)
        side = int((x, y, z)[axis] != 0)
        bs, xs, ys, zs = locate(int(sv) & 0x7FFFFFFF)
        src_c, dst_c = [xs, ys, zs], [x, y, z]
        others = [a for a in range(3) if a != axis]
        assert all(src_c[a] == dst_c[a] for a in others)
        assert src_c[axis] in (1, dims[bs][axis])
        faces.setdefault((b, axis, side), set()).add((bs, src_c[axis]))
    for key, srcs in faces.items():
        assert len(srcs) == 1, key
    assert len(faces) == 6 * len(blocks)
