"""Seeded scene generators for the SPH configurations (host side, numpy).

A dam-break scene is a block of fluid particles on a cubic lattice of spacing
d = 2r, each coordinate jittered uniformly by +-jitter*r from a seeded
Mersenne-Twister stream, sitting in the lower corner of a box whose walls are
`layers` layers of static boundary particles at the same spacing, just outside
the box faces.

Reference semantics that this restates:
  * fluid lattice -- SphWithIO::addFluidCuboid (SphWithIO.cpp:149-194) places a
    lattice of spacing d in a cuboid; here the lattice is given by its point
    counts (nx, ny, nz) directly, with points at lo + (i + 1/2) d, so the
    particle count of every configuration is exact;
  * walls -- SphWithIO::makeCubeSampleParts (SphWithIO.cpp:489-522) samples one
    closed cube surface; the configurations ask for `layers` (2) lattice layers
    outside each face, generated here as a thick shell of lattice points;
  * particle diameter `d` = 2r, smoothRadius_h = 2d (support 4r), spacing_r = d
    (mass = rho0 * spacing_r^3, DFSPH.cpp:88,117), so the reference's kernel
    length m_ker_h = smoothRadius_h / 2 = d (SphBase.h:812).
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Scene:
    fluid_pos: np.ndarray          # (N, 3) float32
    fluid_vel: np.ndarray          # (N, 3) float32
    boundary_pos: np.ndarray       # (Nb, 3) float32
    r: float                       # particle radius
    space_min: tuple
    space_max: tuple
    rho0: float = 1000.0
    phase: np.ndarray = None       # (N,) int32 fluid phase index, or None
    rho0_phases: tuple = (1000.0,)
    meta: dict = field(default_factory=dict)

    @property
    def d(self):
        return 2.0 * self.r

    @property
    def spacing_r(self):
        return 2.0 * self.r

    @property
    def smooth_radius(self):
        return 4.0 * self.r

    @property
    def n_fluid(self):
        return int(self.fluid_pos.shape[0])

    @property
    def n_boundary(self):
        return int(self.boundary_pos.shape[0])


def _rng(seed):
    return np.random.Generator(np.random.MT19937(seed))


def lattice_block(counts, r, lo=(0.0, 0.0, 0.0), jitter=0.1, seed=0):
    """(nx*ny*nz, 3) float32 lattice points at spacing 2r, x fastest, jittered."""
    nx, ny, nz = counts
    d = 2.0 * r
    i = np.arange(nx, dtype=np.float64)
    j = np.arange(ny, dtype=np.float64)
    k = np.arange(nz, dtype=np.float64)
    zz, yy, xx = np.meshgrid(k, j, i, indexing="ij")
    pos = np.stack([lo[0] + (xx.ravel() + 0.5) * d,
                    lo[1] + (yy.ravel() + 0.5) * d,
                    lo[2] + (zz.ravel() + 0.5) * d], axis=1)
    if jitter:
        pos += _rng(seed).uniform(-jitter * r, jitter * r, size=pos.shape)
    return pos.astype(np.float32)


def wall_shell(box, r, layers=2, lo=(0.0, 0.0, 0.0)):
    """Boundary particles: `layers` lattice layers (spacing 2r) outside every
    face of the box [lo, lo+box], as one static rigid solid."""
    d = 2.0 * r
    n = [int(round(box[a] / d)) for a in range(3)]
    rng = [np.arange(-layers, n[a] + layers, dtype=np.int64) for a in range(3)]
    zz, yy, xx = np.meshgrid(rng[2], rng[1], rng[0], indexing="ij")
    xx, yy, zz = xx.ravel(), yy.ravel(), zz.ravel()
    outside = ((xx < 0) | (xx >= n[0]) | (yy < 0) | (yy >= n[1]) | (zz < 0) | (zz >= n[2]))
    pos = np.stack([lo[0] + (xx[outside] + 0.5) * d,
                    lo[1] + (yy[outside] + 0.5) * d,
                    lo[2] + (zz[outside] + 0.5) * d], axis=1)
    return pos.astype(np.float32)


def dam_break(counts, r, box, seed=0, jitter=0.1, layers=2, rho0=1000.0):
    """Fluid block of counts=(nx,ny,nz) particles in the (x-min, y-min, z-min)
    corner of a walled box of size `box` (metres); gravity along -y."""
    fluid = lattice_block(counts, r, jitter=jitter, seed=seed)
    walls = wall_shell(box, r, layers=layers)
    d = 2.0 * r
    margin = (layers + 0.5) * d
    smin = tuple(float(-margin) for _ in range(3))
    smax = tuple(float(box[a] + margin) for a in range(3))
    return Scene(fluid_pos=fluid, fluid_vel=np.zeros_like(fluid), boundary_pos=walls, r=r,
                 space_min=smin, space_max=smax, rho0=rho0, rho0_phases=(rho0,),
                 meta=dict(kind="dam_break", counts=tuple(counts), box=tuple(box), seed=seed))


def box_surface(half, d):
    """Boundary particles on the surface of the box [-half, half] (body
    frame, float32): a lattice of n_a + 1 points per axis with n_a =
    round(2 half_a / d) intervals, the points with an extreme index on some
    axis -- one layer, as SphWithIO::makeCubeSampleParts samples a cube's
    surface (SphWithIO.cpp:489-522)."""
    n = [max(1, int(round(2.0 * half[a] / d))) for a in range(3)]
    ax = [np.arange(n[a] + 1) for a in range(3)]
    zz, yy, xx = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    xx, yy, zz = xx.ravel(), yy.ravel(), zz.ravel()
    surf = (xx == 0) | (xx == n[0]) | (yy == 0) | (yy == n[1]) | (zz == 0) | (zz == n[2])
    pos = np.stack([-half[0] + xx[surf] * (2.0 * half[0] / n[0]),
                    -half[1] + yy[surf] * (2.0 * half[1] / n[1]),
                    -half[2] + zz[surf] * (2.0 * half[2] / n[2])], axis=1)
    return pos.astype(np.float32)


def floating_box(counts, r, box, body_half, body_center, seed=0, jitter=0.1, layers=2, rho0=1000.0):
    """A walled tank whose lower part holds a fluid block of counts=(nx,ny,nz)
    particles, with a box-shaped rigid body (one surface layer of boundary
    particles, solid id 1; the walls are solid 0) at body_center; fluid
    particles closer than d to the body's inside are left out.  The body's
    body-frame particles and its placement are in meta["bodies"]."""
    d = 2.0 * r
    fluid = lattice_block(counts, r, jitter=jitter, seed=seed)
    c = np.asarray(body_center, dtype=np.float64)
    hb = np.asarray(body_half, dtype=np.float64)
    keep = np.any(np.abs(fluid.astype(np.float64) - c) > hb + d, axis=1)
    fluid = np.ascontiguousarray(fluid[keep])
    walls = wall_shell(box, r, layers=layers)
    inner = box_surface(body_half, d)
    body = (inner + np.asarray(body_center, dtype=np.float32)).astype(np.float32)
    margin = (layers + 0.5) * d
    smin = tuple(float(-margin) for _ in range(3))
    smax = tuple(float(box[a] + margin) for a in range(3))
    sid = np.concatenate([np.zeros(len(walls), np.int32), np.ones(len(body), np.int32)])
    return Scene(fluid_pos=fluid, fluid_vel=np.zeros_like(fluid), boundary_pos=np.concatenate([walls, body]), r=r,
                 space_min=smin, space_max=smax, rho0=rho0, rho0_phases=(rho0,),
                 meta=dict(kind="floating_box", counts=tuple(counts), box=tuple(box), seed=seed, solid_id=sid,
                           bodies=[dict(solid_id=1, inner=inner, center=tuple(float(x) for x in body_center),
                                        half=tuple(float(x) for x in body_half))]))


def rayleigh_taylor(counts, r, box, seed=0, jitter=0.1, layers=2, rho_heavy=3000.0, rho_light=1000.0,
                    amplitude=0.02):
    """Two-phase column filling the box: phase 0 (light) below the interface
    y = box_y/2 + amplitude*sin(2 pi x)*sin(2 pi z), phase 1 (heavy) above."""
    pos = lattice_block(counts, r, jitter=jitter, seed=seed)
    walls = wall_shell(box, r, layers=layers)
    x, y, z = pos[:, 0].astype(np.float64), pos[:, 1].astype(np.float64), pos[:, 2].astype(np.float64)
    iface = box[1] / 2 + amplitude * np.sin(2 * np.pi * x) * np.sin(2 * np.pi * z)
    phase = (y > iface).astype(np.int32)
    d = 2.0 * r
    margin = (layers + 0.5) * d
    smin = tuple(float(-margin) for _ in range(3))
    smax = tuple(float(box[a] + margin) for a in range(3))
    return Scene(fluid_pos=pos, fluid_vel=np.zeros_like(pos), boundary_pos=walls, r=r,
                 space_min=smin, space_max=smax, rho0=rho_light, phase=phase,
                 rho0_phases=(rho_light, rho_heavy),
                 meta=dict(kind="rayleigh_taylor", counts=tuple(counts), box=tuple(box), seed=seed))


# Named configurations (sizes from the SPH benchmark configurations).
def config_wcsph_27k(seed=0):
    """27,000-particle WCSPH dam break, r = 0.025 (box widened to 3.0 x 1.6 x
    1.6 m so that the 1.5 m block fits)."""
    return dam_break((30, 30, 30), 0.025, (3.0, 1.6, 1.6), seed=seed)


def config_dfsph_1m(seed=0):
    """1,000,000-particle DFSPH dam break, r = 0.01, 4 x 2 x 2 m box."""
    return dam_break((100, 100, 100), 0.01, (4.0, 2.0, 2.0), seed=seed)


def config_dfsph_2m(seed=0):
    """2,000,000-particle DFSPH dam break, r = 0.008, 200x100x100 block."""
    return dam_break((200, 100, 100), 0.008, (4.0, 2.0, 2.0), seed=seed)


def config_multiphase_500k(seed=0):
    """500,094-particle two-phase Rayleigh-Taylor column (63 x 126 x 63
    lattice, y up), r = 0.0079365 so that it fills a 1 x 2 x 1 m box."""
    r = 0.5 / 63.0
    return rayleigh_taylor((63, 126, 63), r, (1.0, 2.0, 1.0), seed=seed)


def small_dam_break(n=(10, 10, 10), r=0.025, box=None, seed=0):
    if box is None:
        box = (4 * n[0] * r, 2 * n[1] * r, 2 * n[2] * r)
    return dam_break(n, r, box, seed=seed)


def config_batched_dfsph(nscenes=64, seed=0, r=0.01, n_min=1e4, n_max=2e5):
    """Independent dam breaks of uneven size for a batch: N_i drawn
    log-uniformly from [n_min, n_max], block aspect ratios uniform in
    [0.5, 2] per axis (normalised so the lattice holds about N_i particles),
    each block in its own walled box twice its length along x."""
    rng = np.random.default_rng(seed)
    scenes = []
    d = 2.0 * r
    for i in range(nscenes):
        n = float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        a = rng.uniform(0.5, 2.0, 3)
        a = a / np.prod(a) ** (1.0 / 3.0)
        counts = tuple(max(2, int(round(n ** (1.0 / 3.0) * a[k]))) for k in range(3))
        box = (2.0 * counts[0] * d, counts[1] * d, counts[2] * d)
        scenes.append(dam_break(counts, r, box, seed=seed * 1000 + i))
    return scenes

