"""Seeded synthetic pressure-Poisson workloads (the five benchmark configurations
and a local-mesh-refinement one).

No public dataset is involved: every right-hand side is the discrete
divergence of a seeded velocity field, computed the way calmas does it
(src_v70/press.for:48-58: b = div(u)/dt with dt = 1; the L_LSM branch scales
by the cell volume), with boundary-normal wall velocities zero so the
all-Neumann problems are compatible.  Seeds: numpy PCG64, 1000 + config
index (and +17 for the "previous solve" field of configuration 2).

Every generator takes `resolve`, passed on to topology.from_extents: None
finds block neighbours with the library, a callable finds them without it.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import topology
from .mg import host_field, interior, with_ghost

WALL, PER = topology.WALL, topology.PERIODIC


@dataclass
class Problem:
    name: str
    blocks: list
    ngrid: int
    b: List[np.ndarray]                    # host fields (ttc, pl ghosts)
    p0: List[np.ndarray]                   # host fields
    dens: Optional[List[np.ndarray]] = None  # host fields (L_LSM only)
    var_coef: bool = False
    meta: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return int(sum(d.n[0] * d.n[1] * d.n[2] for d in self.blocks))


def divergence(ux, uy, uz, h, periodic=(False, False, False)):
    """Cell divergence of face velocities.

    ux has shape (nz, ny, nx+1) (faces x_i, i = 0..nx), uy (nz, ny+1, nx),
    uz (nz+1, ny, nx).  Faces on a wall are forced to zero (the wall face the
    reference never updates, localparameters.for:187-192); on a periodic axis
    the last face equals the first."""
    ux = ux.copy(); uy = uy.copy(); uz = uz.copy()
    if periodic[0]:
        ux[:, :, -1] = ux[:, :, 0]
    else:
        ux[:, :, 0] = 0.0; ux[:, :, -1] = 0.0
    if periodic[1]:
        uy[:, -1, :] = uy[:, 0, :]
    else:
        uy[:, 0, :] = 0.0; uy[:, -1, :] = 0.0
    if periodic[2]:
        uz[-1] = uz[0]
    else:
        uz[0] = 0.0; uz[-1] = 0.0
    return (ux[:, :, 1:] - ux[:, :, :-1]) / h[0] + (uy[:, 1:, :] - uy[:, :-1, :]) / h[1] + \
        (uz[1:] - uz[:-1]) / h[2]


def _uniform_velocity(rng, n):
    nx, ny, nz = n
    return (rng.uniform(-1.0, 1.0, (nz, ny, nx + 1)), rng.uniform(-1.0, 1.0, (nz, ny + 1, nx)),
            rng.uniform(-1.0, 1.0, (nz + 1, ny, nx)))


def _split(global_field, blocks):
    """Scatter a global (NZ, NY, NX) cell field into block host fields."""
    out = []
    for d in blocks:
        a = host_field(d)
        o = d.origin
        interior(a, d)[...] = global_field[o[2]:o[2] + d.n[2], o[1]:o[1] + d.n[1], o[0]:o[0] + d.n[0]]
        out.append(a)
    return out


def gather(fields, blocks):
    """Inverse of the scatter into blocks: the global (NZ, NY, NX) cell field
    of block host fields placed at their origins."""
    NX = max(d.origin[0] + d.n[0] for d in blocks)
    NY = max(d.origin[1] + d.n[1] for d in blocks)
    NZ = max(d.origin[2] + d.n[2] for d in blocks)
    g = np.zeros((NZ, NY, NX))
    for a, d in zip(fields, blocks):
        o = d.origin
        g[o[2]:o[2] + d.n[2], o[1]:o[1] + d.n[1], o[0]:o[0] + d.n[0]] = interior(a, d)
    return g


def config1(seed: int = 1001, n: int = 64, ngrid: int = 4, resolve=None) -> Problem:
    """Single block n^3, h = 1/n, walls on all faces, zero initial guess."""
    rng = np.random.Generator(np.random.PCG64(seed))
    h = (1.0 / n,) * 3
    blocks = topology.block_grid((1, 1, 1), (n, n, n), [WALL] * 6, h, ngrid, resolve=resolve)
    b = divergence(*_uniform_velocity(rng, (n, n, n)), h)
    return Problem("config1", blocks, ngrid, _split(b, blocks), [host_field(d) for d in blocks],
                   meta=dict(seed=seed))


def _config2_rhs(seed, N, h):
    rng = np.random.Generator(np.random.PCG64(seed))
    ux, uy, uz = _uniform_velocity(rng, (N, N, N))
    b = divergence(ux, uy, uz, h, periodic=(True, False, False))
    xc = (np.arange(N) + 0.5) * h[0]
    yc = (np.arange(N) + 0.5) * h[1]
    b = b + (np.sin(2 * np.pi * xc)[None, None, :] * np.cos(2 * np.pi * yc)[None, :, None])
    return b


def config2(seed: int = 1002, nb: int = 2, n: int = 96, ngrid: int = 6, p0: Optional[np.ndarray] = None,
            resolve=None) -> Problem:
    """(nb*n)^3 as nb^3 blocks of n^3; periodic in x, walls in y and z.

    b = div u of a U(-1,1) velocity (periodic in x) plus sin(2 pi x)cos(2 pi y)
    (zero discrete sum, so the problem stays compatible).  The initial guess
    is a converged pressure of the independent seed `seed + 15` problem
    (1017 for the default seed); pass it as `p0` (a global (N,N,N) array) or
    use `config2_previous_rhs` to build that problem."""
    N = nb * n
    h = (1.0 / N,) * 3
    bc = [PER, PER, WALL, WALL, WALL, WALL]
    blocks = topology.block_grid((nb, nb, nb), (n, n, n), bc, h, ngrid, resolve=resolve)
    b = _config2_rhs(seed, N, h)
    pinit = [host_field(d) for d in blocks]
    if p0 is not None:
        for d, a in zip(blocks, pinit):
            o = d.origin
            interior(a, d)[...] = p0[o[2]:o[2] + d.n[2], o[1]:o[1] + d.n[1], o[0]:o[0] + d.n[0]]
    return Problem("config2", blocks, ngrid, _split(b, blocks), pinit, meta=dict(seed=seed, prev_seed=seed + 15))


def config2_previous_rhs(seed: int = 1017, nb: int = 2, n: int = 96) -> np.ndarray:
    N = nb * n
    return _config2_rhs(seed, N, (1.0 / N,) * 3)


def spectral_velocity(rng, shape, box, kmin=1.0, kmax=64.0):
    """A real field with Fourier amplitudes |k|^(-5/3) on kmin <= |k| <= kmax,
    uniform random phases, unit RMS.  shape = (nz, ny, nx); box = (Lz, Ly, Lx);
    |k| counts waves per unit length."""
    nz, ny, nx = shape
    kz = np.fft.fftfreq(nz, d=box[0] / nz)
    ky = np.fft.fftfreq(ny, d=box[1] / ny)
    kx = np.fft.rfftfreq(nx, d=box[2] / nx)
    kk = np.sqrt(kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2)
    amp = np.where((kk >= kmin) & (kk <= kmax), np.power(np.maximum(kk, 1e-30), -5.0 / 3.0), 0.0)
    phase = rng.uniform(0.0, 2 * np.pi, amp.shape)
    spec = amp * np.exp(1j * phase)
    f = np.fft.irfftn(spec, s=shape, axes=(0, 1, 2))
    f /= np.sqrt(np.mean(f * f))
    return f


def config3(seed: int = 1003, nblk=(4, 2, 2), n: int = 128, ngrid: int = 7, resolve=None) -> Problem:
    """512x256x256 cells as 4x2x2 blocks of 128^3, all walls, spectral velocity."""
    rng = np.random.Generator(np.random.PCG64(seed))
    NX, NY, NZ = nblk[0] * n, nblk[1] * n, nblk[2] * n
    hh = 1.0 / max(NY, NZ)
    h = (hh, hh, hh)
    blocks = topology.block_grid(nblk, (n, n, n), [WALL] * 6, h, ngrid, resolve=resolve)
    box = (NZ * hh, NY * hh, NX * hh)
    comps = []
    for _ in range(3):
        comps.append(spectral_velocity(rng, (NZ, NY, NX), box))
    fx, fy, fz = comps
    ux = np.concatenate([fx, fx[:, :, :1]], axis=2)
    uy = np.concatenate([fy, fy[:, :1, :]], axis=1)
    uz = np.concatenate([fz, fz[:1]], axis=0)
    del comps, fx, fy, fz
    b = divergence(ux, uy, uz, h)
    return Problem("config3", blocks, ngrid, _split(b, blocks), [host_field(d) for d in blocks],
                   meta=dict(seed=seed))


def config4(seed: int = 1004, nblocks: int = 27, ngrid: int = 4, choices=(32, 48, 64, 96, 128),
            resolve=None) -> Problem:
    """27 independent wall-bounded blocks of seeded uneven sizes, h = 1/64."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = [tuple(int(v) for v in rng.choice(choices, size=3)) for _ in range(nblocks)]
    h = (1.0 / 64,) * 3
    blocks = topology.independent_blocks(sizes, h, ngrid, resolve=resolve)
    bs = []
    for d in blocks:
        n = (d.n[0], d.n[1], d.n[2])
        a = host_field(d)
        interior(a, d)[...] = divergence(*_uniform_velocity(rng, n), h)
        bs.append(a)
    return Problem("config4", blocks, ngrid, bs, [host_field(d) for d in blocks], meta=dict(seed=seed, sizes=sizes))


def heaviside(phi, eps):
    """Smoothed Heaviside of src_v70/lsm.for:1533-1540."""
    Hs = np.where(phi < -eps, 0.0, np.where(phi > eps, 1.0, 0.0))
    band = np.abs(phi) <= eps
    Hs = np.where(band, 0.5 * (1.0 + phi / eps + np.sin(np.pi * phi / eps) / np.pi), Hs)
    return Hs


def config5(seed: int = 1005, n: int = 256, ngrid: int = 8, rho_l: float = 1000.0, rho_g: float = 1.0,
            resolve=None) -> Problem:
    """Two-phase variable-coefficient problem: single block n^3, density from a
    seeded sphere level set (heavy fluid outside), L_LSM coefficients."""
    rng = np.random.Generator(np.random.PCG64(seed))
    hh = 1.0 / n
    h = (hh, hh, hh)
    c = rng.uniform(0.3, 0.7, 3)
    blocks = topology.block_grid((1, 1, 1), (n, n, n), [WALL] * 6, h, ngrid, resolve=resolve)
    xc = (np.arange(n) + 0.5) * hh
    phi = np.sqrt((xc[None, None, :] - c[0]) ** 2 + (xc[None, :, None] - c[1]) ** 2 +
                  (xc[:, None, None] - c[2]) ** 2) - 0.2
    rho = rho_g + (rho_l - rho_g) * heaviside(phi, 1.5 * hh)
    div = divergence(*_uniform_velocity(rng, (n, n, n)), h)
    sup = div * (hh * hh * hh)  # press.for:53-55 (dt = 1)
    d = blocks[0]
    return Problem("config5", blocks, ngrid, _split(sup, blocks), [host_field(d)], dens=_split(rho, blocks),
                   var_coef=True, meta=dict(seed=seed, centre=c.tolist()))


def smooth_pressure(rng, nmodes: int = 24, kmax: float = 4.0):
    """A seeded smooth pressure: nmodes cosines cos(2 pi k.x + phase) with
    integer wave vectors 1 <= |k| <= kmax and amplitude |k|^(-5/3); returns
    p(x, y, z) for cell-centre coordinate arrays."""
    ks, amps, phases = [], [], []
    while len(ks) < nmodes:
        k = rng.integers(-int(kmax), int(kmax) + 1, 3)
        kn = float(np.sqrt((k * k).sum()))
        if 1.0 <= kn <= kmax:
            ks.append(k.astype(np.float64))
            amps.append(kn ** (-5.0 / 3.0))
            phases.append(rng.uniform(0.0, 2.0 * np.pi))

    def p(x, y, z):
        out = np.zeros(np.broadcast(x, y, z).shape)
        for k, a, ph in zip(ks, amps, phases):
            out += a * np.cos(2.0 * np.pi * (k[0] * x + k[1] * y + k[2] * z) + ph)
        return out
    return p


def config6(seed: int = 1006, nblk=(4, 2, 2), n: int = 64, ngrid_input: int = 6, refined=(1, 2),
            resolve=None) -> Problem:
    """Local mesh refinement (LMR = 2): 4x2x2 blocks of n^3 unrefined cells
    (h = 1/(2n)), those of x index in `refined` refined by 2 (2n cells a side
    at h/2): 8 x 64^3 + 8 x 128^3 = 18.9M cells, walls, 7 levels.

    The operator with refinement is not symmetric and its left null vector is
    not constant, so a divergence right-hand side is not compatible.  The
    right-hand side is b = A p of the seeded smooth pressure meta["p_exact"]
    (host fields), made by each solver's own operator: `b` is None until
    `manufacture` fills it."""
    rng = np.random.Generator(np.random.PCG64(seed))
    hh = 1.0 / (nblk[1] * n)
    blocks = topology.block_grid(nblk, (n, n, n), [WALL] * 6, (hh,) * 3, ngrid_input, resolve=resolve)
    rdiv = [2 if (b % nblk[0]) in refined else 1 for b in range(len(blocks))]
    topology.refine(blocks, rdiv, ngrid_input)
    pf = smooth_pressure(rng)
    pex = []
    for d in blocks:
        a = host_field(d)
        x = (d.origin[0] + np.arange(d.n[0]) + 0.5) * d.h[0]
        y = (d.origin[1] + np.arange(d.n[1]) + 0.5) * d.h[1]
        z = (d.origin[2] + np.arange(d.n[2]) + 0.5) * d.h[2]
        interior(a, d)[...] = pf(x[None, None, :], y[None, :, None], z[:, None, None])
        pex.append(a)
    return Problem("config6", blocks, ngrid_input + 1, None, [host_field(d) for d in blocks],
                   meta=dict(seed=seed, rdiv=rdiv, p_exact=pex))


def manufacture(prob: Problem, residual_of):
    """Fills prob.b = A p_exact for a manufactured workload; residual_of(p)
    returns the interior residual b - A p of b = 0 per block (canonical
    (nz, ny, nx) arrays)."""
    if prob.b is not None:
        return prob
    r = residual_of(prob.meta["p_exact"])
    prob.b = []
    for d, x in zip(prob.blocks, r):
        a = host_field(d)
        interior(a, d)[...] = -x
        prob.b.append(a)
    return prob


CONFIGS = {1: config1, 2: config2, 3: config3, 4: config4, 5: config5, 6: config6}
