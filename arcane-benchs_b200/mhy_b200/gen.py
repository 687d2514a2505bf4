"""Seeded generators for meshes and initial states (the inputs of every run).

MaHyCo builds its mesh with Arcane's Cartesian generator and its initial state
with test-case services (mahyco/src/casTest/SOD/SODService.cc:11-126,
mahyco/src/casTest/SEDOV/SEDOVService.cc:39-131).  Neither is available here, so
the same kind of input is generated on the host, deterministically, and the
identical arrays feed both the CPU oracle and the GPU.

Random numbers come from SplitMix64 (Steele, Lea & Flood 2014): state s_i =
seed + i * 0x9E3779B97F4A7C15, output = mix(s_i), uniform double = top 53 bits
* 2^-53.

Layouts (all float64, C order):
  node coordinates  (N, 3), node id = i + (nx+1)*(j + (ny+1)*k)
  per-cell arrays   (nenv, C), cell id = i + nx*(j + ny*k)
  node velocity     (N, 3)
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """n outputs of SplitMix64 starting at stream position `offset`."""
    with np.errstate(over="ignore"):
        i = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, n: int, offset: int = 0) -> np.ndarray:
    return (splitmix64(seed, n, offset) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


# Boundary-condition surfaces and types (MahycoAnnexe.cc:183-251, TypesMahyco.h:9-18)
XMIN, XMAX, YMIN, YMAX, ZMIN, ZMAX = range(6)
VX, VY, VZ = range(3)
WALLS = ((XMIN, VX, 0.0), (XMAX, VX, 0.0), (YMIN, VY, 0.0), (YMAX, VY, 0.0),
         (ZMIN, VZ, 0.0), (ZMAX, VZ, 0.0))


@dataclasses.dataclass
class Options:
    """Mahyco.axl / RemapADI.axl options with the reference defaults
    (Mahyco.axl:296-313, RemapADI.axl:139-177) and the deck values of
    mahyco/data/Data.1.arc:59-104."""
    cfl: float = 0.3
    threshold: float = 1.0e-10
    deltat_init: float = 1.0e-5
    deltat_min: float = 1.0e-8
    deltat_max: float = 0.01
    final_time: float = 0.2
    longueur_caracteristique: int = 0       # 0 racine-cubique-volume, 1 faces-opposees
    pseudo_centree: int = 0
    ordre_projection: int = 2
    projection_limiteur_id: int = 0         # 0 minmod, 1 superBee, 2 vanLeer
    boundary_conditions: tuple = WALLS
    precision: int = 0                      # device only: 0 FP64, 1 mixed (FP32 remap evaluation)
    eos: tuple = ()                         # per environment: 0 PerfectGas (default), 1 StiffenedGas
    limit_tension: tuple = ()               # per environment: StiffenedGas limit-tension (StiffenedGasEOS.axl:104)
    with_newton: int = 0                    # energy update by Newton iterations (Mahyco.axl:308)
    schema_csts: int = 0                    # the CSTS time scheme (Mahyco.axl:238)
    pente_borne: int = 0                    # projection-pente-borne (RemapADI.axl:167)
    pente_borne_debar_fix: int = 0          # projection-pente-borne-debar-fix: 0, 1 or 2 (RemapADI.axl:171)
    pente_borne_mixte: int = 0              # projection-pente-borne-mixte (RemapADI.axl:155)
    limiteur_pure_id: int = 0               # projection-limiteur-pure-id (RemapADI.axl:163)
    conservation_energie_totale: int = 0    # conservation-energie-totale (RemapADI.axl:151)


@dataclasses.dataclass
class Case:
    """One problem instance: mesh, environments, initial state, options."""
    name: str
    nx: int
    ny: int
    nz: int
    coords: np.ndarray        # (N,3)
    gamma: np.ndarray         # (nenv,)
    fracvol: np.ndarray       # (nenv, C)
    density: np.ndarray       # (nenv, C)
    pressure: np.ndarray      # (nenv, C)
    velocity: np.ndarray      # (N,3)
    options: Options
    cycles: int

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def nnodes(self) -> int:
        return (self.nx + 1) * (self.ny + 1) * (self.nz + 1)

    @property
    def nenv(self) -> int:
        return int(self.gamma.shape[0])


def cartesian_nodes(nx, ny, nz, lx, ly, lz, jitter=0.0, seed=0, origin=(0.0, 0.0, 0.0)):
    """Node coordinates of an nx*ny*nz hex grid on [0,lx]x[0,ly]x[0,lz].

    jitter: amplitude as a fraction of the cell width; every node on one of the
    six boundary planes keeps its exact lattice position, so that the boundary
    groups found by coordinate threshold (MahycoAnnexe.cc:212-217) are the
    lattice planes."""
    hx, hy, hz = lx / nx, ly / ny, lz / nz
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    i = i.ravel(); j = j.ravel(); k = k.ravel()
    x = origin[0] + i * hx
    y = origin[1] + j * hy
    z = origin[2] + k * hz
    if jitter > 0.0:
        n = x.size
        u = uniform01(seed, 3 * n).reshape(n, 3)
        d = (2.0 * u - 1.0) * jitter
        inner = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
        x = x + np.where(inner, d[:, 0] * hx, 0.0)
        y = y + np.where(inner, d[:, 1] * hy, 0.0)
        z = z + np.where(inner, d[:, 2] * hz, 0.0)
    return np.ascontiguousarray(np.stack([x, y, z], axis=1))


def cell_centres(coords, nx, ny, nz):
    c = coords.reshape(nz + 1, ny + 1, nx + 1, 3)
    s = (c[:-1, :-1, :-1] + c[:-1, :-1, 1:] + c[:-1, 1:, :-1] + c[:-1, 1:, 1:]
         + c[1:, :-1, :-1] + c[1:, :-1, 1:] + c[1:, 1:, :-1] + c[1:, 1:, 1:]) * 0.125
    return s.reshape(-1, 3)


def sod(nx=100, ny=5, nz=5, lx=1.0, ly=0.05, lz=0.05, axis=0, gamma=1.4, cycles=200,
        rho=(1.0, 0.125), p=(1.0, 0.1), jitter=0.0, seed=0, options=None) -> Case:
    """Sod shock tube (SODService.cc:11-40): left rho/p for centre < half the
    domain along `axis`, right state elsewhere, at rest, one ideal gas."""
    coords = cartesian_nodes(nx, ny, nz, lx, ly, lz, jitter, seed)
    xc = cell_centres(coords, nx, ny, nz)[:, axis]
    half = (lx, ly, lz)[axis] * 0.5
    left = xc < half
    C = nx * ny * nz
    dens = np.where(left, rho[0], rho[1]).reshape(1, C)
    pres = np.where(left, p[0], p[1]).reshape(1, C)
    return Case("sod", nx, ny, nz, coords, np.array([gamma]), np.ones((1, C)), dens, pres,
                np.zeros_like(coords), options or Options(), cycles)


def sedov(n=128, length=1.2, jitter=0.01, seed=1, gamma=1.4, rho=1.0, e_amb=1.0e-12,
          energy=0.979264, deposit_cells=2, cycles=500, options=None) -> Case:
    """Sedov point blast in the octant [0,L]^3 with symmetry planes x=y=z=0.

    `energy` is deposited uniformly (per unit mass, nominal volume h^3) in the
    deposit_cells^3 block of cells at the origin corner; ambient e = e_amb.
    The state is given as (rho, p = (gamma-1) rho e), as the reference's test
    case does before its EOS initialisation (SEDOVService.cc:43-77, E:20-32)."""
    nx = ny = nz = n
    coords = cartesian_nodes(n, n, n, length, length, length, jitter, seed)
    C = n ** 3
    h = length / n
    e = np.full(C, e_amb)
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    corner = ((i < deposit_cells) & (j < deposit_cells) & (k < deposit_cells)).ravel()
    e[corner] = energy / (deposit_cells ** 3 * rho * h ** 3)
    dens = np.full((1, C), rho)
    pres = ((gamma - 1.0) * rho * e).reshape(1, C)
    return Case("sedov", nx, ny, nz, coords, np.array([gamma]), np.ones((1, C)), dens, pres,
                np.zeros_like(coords), options or Options(), cycles)


def _fractions_by_subsampling(nx, ny, nz, lx, ly, lz, inside_fn, sub=4):
    """Volume fraction of material A per cell from sub^3 sub-cell centres."""
    hx, hy, hz = lx / nx, ly / ny, lz / nz
    frac = np.zeros((nz, ny, nx))
    offs = (np.arange(sub) + 0.5) / sub
    xs = (np.arange(nx)[None, None, :] + 0.0) * hx
    ys = (np.arange(ny)[None, :, None] + 0.0) * hy
    zs = (np.arange(nz)[:, None, None] + 0.0) * hz
    for a in offs:
        for b in offs:
            for c in offs:
                frac += inside_fn(xs + a * hx, ys + b * hy, zs + c * hz)
    return (frac / sub ** 3).ravel()


def two_material(nx=256, ny=128, nz=128, lx=1.0, ly=0.5, lz=0.5, seed=2, cycles=1000,
                 amp=0.02, modes=4, options=None) -> Case:
    """Gas A (gamma 1.4, rho 1, p 1) for x < x_I(y,z), gas B (gamma 1.67, rho 0.2,
    p 0.1) elsewhere; x_I = 0.5 + sum_m (amp/modes) sin(2 pi m y/ly + phi_m)
    sin(2 pi m z/lz + psi_m), phases from the seed; fractions by 4^3 sampling."""
    ph = uniform01(seed, 2 * modes) * 2.0 * math.pi

    def inside_a(x, y, z):
        xi = 0.5 * lx + sum((amp / modes) * np.sin(2 * math.pi * m * y / ly + ph[2 * (m - 1)])
                            * np.sin(2 * math.pi * m * z / lz + ph[2 * (m - 1) + 1])
                            for m in range(1, modes + 1))
        return (x < xi).astype(np.float64)

    fa = _fractions_by_subsampling(nx, ny, nz, lx, ly, lz, inside_a)
    return _two_env_case("two_material", nx, ny, nz, lx, ly, lz, fa, cycles, options)


def _two_env_case(name, nx, ny, nz, lx, ly, lz, fa, cycles, options):
    coords = cartesian_nodes(nx, ny, nz, lx, ly, lz)
    C = nx * ny * nz
    fb = 1.0 - fa
    fr = np.stack([fa, fb])
    fr[fr < 0.0] = 0.0
    dens = np.stack([np.where(fa > 0, 1.0, 0.0), np.where(fb > 0, 0.2, 0.0)])
    pres = np.stack([np.where(fa > 0, 1.0, 0.0), np.where(fb > 0, 0.1, 0.0)])
    return Case(name, nx, ny, nz, coords, np.array([1.4, 1.67]), fr, dens, pres,
                np.zeros_like(coords), options or Options(), cycles)


def three_material(nx=48, ny=16, nz=16, lx=1.0, ly=0.3, lz=0.3, seed=6, cycles=100, amp=0.03,
                   radius=0.08, options=None) -> Case:
    """Three ideal gases: A (gamma 1.4, rho 1, p 1) for x < x_I(y,z), B (gamma
    1.67, rho 0.3, p 0.2) beyond, and a cylinder of C (gamma 1.3, rho 0.6,
    p 0.05) along z of the given radius centred on the interface at y = ly/2,
    so that cells hold one, two or all three environments.  x_I = lx/2 +
    amp sin(2 pi y/ly + phi) cos(2 pi z/lz + psi), phases from the seed;
    fractions by 4^3 sampling."""
    ph = uniform01(seed, 2) * 2.0 * math.pi
    sub = 4
    hx, hy, hz = lx / nx, ly / ny, lz / nz
    frac = np.zeros((3, nz, ny, nx))
    offs = (np.arange(sub) + 0.5) / sub
    xs = np.arange(nx)[None, None, :] * hx
    ys = np.arange(ny)[None, :, None] * hy
    zs = np.arange(nz)[:, None, None] * hz
    for a in offs:
        for b in offs:
            for c in offs:
                x, y, z = xs + a * hx, ys + b * hy, zs + c * hz
                xi = 0.5 * lx + amp * np.sin(2 * math.pi * y / ly + ph[0]) * np.cos(2 * math.pi * z / lz + ph[1])
                inc = (x - 0.5 * lx) ** 2 + (y - 0.5 * ly) ** 2 < radius ** 2
                isa = (x < xi) & ~inc
                frac[0] += isa
                frac[1] += ~isa & ~inc
                frac[2] += inc
    fr = (frac / sub ** 3).reshape(3, -1)
    coords = cartesian_nodes(nx, ny, nz, lx, ly, lz)
    rho = (1.0, 0.3, 0.6)
    p = (1.0, 0.2, 0.05)
    dens = np.stack([np.where(fr[k] > 0, rho[k], 0.0) for k in range(3)])
    pres = np.stack([np.where(fr[k] > 0, p[k], 0.0) for k in range(3)])
    return Case("three_material", nx, ny, nz, coords, np.array([1.4, 1.67, 1.3]), fr, dens, pres,
                np.zeros_like(coords), options or Options(), cycles)


def _real_sph_harm(l, m, theta, phi):
    """Real spherical harmonic Y_lm (unnormalised associated Legendre form)."""
    from scipy.special import lpmv  # scipy is in the image
    x = np.cos(theta)
    plm = lpmv(abs(m), l, x)
    if m > 0:
        return plm * np.cos(m * phi)
    if m < 0:
        return plm * np.sin(-m * phi)
    return plm


def sphere_inclusion(nx=384, ny=384, nz=192, lx=1.0, ly=1.0, lz=0.5, radius=0.25, amp=0.01,
                     seed=4, cycles=200, options=None) -> Case:
    """Sphere of gas B centred at the box centre in gas A; radius perturbed by 8
    real spherical-harmonic modes (l=2..3) of amplitude `amp`, coefficients from the seed."""
    lm = [(2, -2), (2, -1), (2, 0), (2, 1), (2, 2), (3, -1), (3, 0), (3, 1)]
    coef = (2.0 * uniform01(seed, len(lm)) - 1.0)
    cx, cy, cz = lx / 2, ly / 2, lz / 2

    def inside_a(x, y, z):
        dx, dy, dz = x - cx, y - cy, z - cz
        r = np.sqrt(dx * dx + dy * dy + dz * dz)
        theta = np.arccos(np.clip(dz / np.maximum(r, 1e-300), -1, 1))
        phi = np.arctan2(dy, dx)
        pert = sum(c * _real_sph_harm(l, m, theta, phi) for c, (l, m) in zip(coef, lm))
        return (r >= radius * (1.0 + amp * pert)).astype(np.float64)

    fa = _fractions_by_subsampling(nx, ny, nz, lx, ly, lz, inside_a)
    return _two_env_case("sphere_inclusion", nx, ny, nz, lx, ly, lz, fa, cycles, options)


def batched(count=64, seed=3, side_lo=32, side_hi=96, cycles=300):
    """Independent instances with uneven cubic meshes on the unit cube: even
    index Sod along x, odd index Sedov-like corner deposit; gamma ~ U[1.3,1.7],
    left/right density ratio log-uniform in [2,20]."""
    u = uniform01(seed, 4 * count).reshape(count, 4)
    cases = []
    for b in range(count):
        s = side_lo + int(u[b, 0] * (side_hi - side_lo + 1))
        g = 1.3 + 0.4 * u[b, 1]
        ratio = math.exp(math.log(2.0) + u[b, 2] * (math.log(20.0) - math.log(2.0)))
        if b % 2 == 0:
            c = sod(s, s, s, 1.0, 1.0, 1.0, gamma=g, cycles=cycles, rho=(1.0, 1.0 / ratio), p=(1.0, 0.1))
        else:
            c = sedov(n=s, length=1.0, jitter=0.0, gamma=g, cycles=cycles, energy=0.979264 / ratio)
        c.name = f"batch{b}"
        cases.append(c)
    return cases
