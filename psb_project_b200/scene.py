"""Scene description: the Python mirror of ``psb_scene`` (include/psb.h) and
the synthetic dam-break scenes the benchmarks and tests run.

The reference builds scenes interactively (Qt dialogs, EmitterBox lattices:
src/Kernel/Emitters/EmitterBox.cpp:29-47, spacing 2*particleRadius) and
keeps material parameters in per-particle arrays filled from
SimulationData_SPHSystem (SimulationData_SPHSystem.cpp:5-16). Here a scene
is one uniform parameter set plus one or more lattice blocks.

Conventions fixed here (the scene text leaves them open):
  * y is up and gravity is (0, -9.81, 0), as the reference's PCISPH
    kernel hard-codes it (PciSphSystem_Kernel.cu:168);
  * the box spans [0, L] on each axis and the lattice block sits in the
    (0, 0, 0) corner, first particle at spacing/2 from the walls;
  * the grid covers the box plus one cell on each side;
  * the cell edge is (1 + skin) h rounded up to the next float, so the
    27-cell walk sees every pair the list keeps; the skin defaults to 0
    (config scenes may set one so that pairs closing in during a step's
    predictions are listed: at dt = 5e-4 the 1M dam break converges the same
    without, at 28% less gather work); reference-profile parity scenes use a
    cell of float(h), exactly as PCI_SPHSystem::_initialize passes
    getInteractionRadius() to createGrid (PciSphSystem.cpp:143);
  * where the text gives no particle mass, the mass puts a filled lattice
    exactly at rest density (lattice_mass); rho0 * spacing^3 would leave
    it 0.98% over rest density at h = 2 spacing, a whole eta of 1%;
  * config-profile walls: mirror ghosts across the faces for density and
    pressure, and a penalty outside the faces (wall_k = 0.5/dt^2, wall_c =
    sqrt(wall_k), damping ratio 0.5), as C0 states for WCSPH; PCISPH also
    projects after every step into [Min + r, Max - r] with the normal
    velocity removed, as the reference's BoxCollision does;
  * the particle (wall) radius is spacing/2;
  * config-profile PCISPH smooths the committed velocities with XSPH,
    factor 0.25 (Monaghan 1989): at h = 2 spacing the poly6 density of a
    moving, disordered particle set is noisy, and without it the
    particle-scale velocity noise compresses pairs by ~10% within one step
    (the corrector's first error), against ~4% with it; the mean correction
    count of the 1M dam break drops from 13.4 to 9.4;
  * C2 states no time step: dt = 5e-4 s, the C1 step (1e-3 s at h = 0.02 m)
    scaled with h as a CFL bound is, and the step C4 uses at h = 0.008 m.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

PROFILE_REF = 0
PROFILE_CONFIG = 1
WCSPH = 0
PCISPH = 1
DEM = 2
WARM_ZERO = 0
WARM_PREVIOUS = 1
WARM_LEARNED = 2


class PsbScene(ctypes.Structure):
    """Binary layout of ``psb_scene`` (include/psb.h)."""

    _fields_ = [
        ("n_max", ctypes.c_int32),
        ("box_min", ctypes.c_float * 3),
        ("box_max", ctypes.c_float * 3),
        ("grid_min", ctypes.c_float * 3),
        ("cell", ctypes.c_float),
        ("dims", ctypes.c_int32 * 3),
        ("h", ctypes.c_double),
        ("mass", ctypes.c_double),
        ("rho0", ctypes.c_double),
        ("k", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("sigma", ctypes.c_double),
        ("l", ctypes.c_double),
        ("particle_radius", ctypes.c_float),
        ("dt", ctypes.c_float),
        ("gravity", ctypes.c_float * 3),
        ("profile", ctypes.c_int32),
        ("method", ctypes.c_int32),
        ("min_iters", ctypes.c_int32),
        ("max_iters", ctypes.c_int32),
        ("eta", ctypes.c_double),
        ("wall_k", ctypes.c_double),
        ("wall_c", ctypes.c_double),
        ("nbr_cap", ctypes.c_int32),
        ("warm_start", ctypes.c_int32),
        ("spacing", ctypes.c_double),
        ("skin", ctypes.c_double),
        ("xsph", ctypes.c_double),
        ("dem_spring", ctypes.c_double),
        ("dem_damping", ctypes.c_double),
        ("dem_shear", ctypes.c_double),
        ("dem_attraction", ctypes.c_double),
    ]


@dataclasses.dataclass
class Block:
    """A lattice block: counts per axis, spacing, corner, jitter, seed, first id."""

    nxyz: Tuple[int, int, int]
    spacing: float
    origin: Tuple[float, float, float]
    jitter: float
    seed: int
    id0: int = 0

    @property
    def n(self) -> int:
        return self.nxyz[0] * self.nxyz[1] * self.nxyz[2]


@dataclasses.dataclass
class Scene:
    n: int
    box_min: Tuple[float, float, float]
    box_max: Tuple[float, float, float]
    grid_min: Tuple[float, float, float]
    cell: float
    dims: Tuple[int, int, int]
    h: float
    mass: float
    rho0: float = 1000.0
    k: float = 3.0
    mu: float = 0.01
    sigma: float = 0.0
    l: float = 7.065
    particle_radius: float = 0.005
    dt: float = 1e-3
    gravity: Tuple[float, float, float] = (0.0, -9.81, 0.0)
    profile: int = PROFILE_CONFIG
    method: int = PCISPH
    min_iters: int = 3
    max_iters: int = 50
    eta: float = 0.01
    wall_k: float = 0.0
    wall_c: float = 0.0
    nbr_cap: int = 128
    warm_start: int = WARM_ZERO
    spacing: float = 0.0
    skin: float = 0.0
    xsph: float = 0.0
    dem_spring: float = 0.0
    dem_damping: float = 0.0
    dem_shear: float = 0.0
    dem_attraction: float = 0.0
    blocks: List[Block] = dataclasses.field(default_factory=list)
    name: str = ""
    steps: int = 0

    def to_c(self) -> PsbScene:
        s = PsbScene()
        s.n_max = self.n
        s.box_min[:] = [float(v) for v in self.box_min]
        s.box_max[:] = [float(v) for v in self.box_max]
        s.grid_min[:] = [float(v) for v in self.grid_min]
        s.cell = self.cell
        s.dims[:] = [int(v) for v in self.dims]
        s.h, s.mass, s.rho0, s.k = self.h, self.mass, self.rho0, self.k
        s.mu, s.sigma, s.l = self.mu, self.sigma, self.l
        s.particle_radius, s.dt = self.particle_radius, self.dt
        s.gravity[:] = [float(v) for v in self.gravity]
        s.profile, s.method = self.profile, self.method
        s.min_iters, s.max_iters, s.eta = self.min_iters, self.max_iters, self.eta
        s.wall_k, s.wall_c = self.wall_k, self.wall_c
        s.nbr_cap, s.warm_start = self.nbr_cap, self.warm_start
        s.spacing = self.spacing
        s.skin = self.skin
        s.xsph = self.xsph
        s.dem_spring, s.dem_damping = self.dem_spring, self.dem_damping
        s.dem_shear, s.dem_attraction = self.dem_shear, self.dem_attraction
        return s

    def replace(self, **kw) -> "Scene":
        return dataclasses.replace(self, **kw)


def f32(x: float) -> float:
    return float(np.float32(x))


def cell_for(h: float, exact_reference: bool) -> float:
    """float(h), or the smallest float >= h (see module docstring)."""
    c = np.float32(h)
    if not exact_reference and float(c) < h:
        c = np.nextafter(c, np.float32(np.inf), dtype=np.float32)
    return float(c)


def grid_for(box_min, box_max, cell: float) -> Tuple[Tuple[float, ...], Tuple[int, ...]]:
    """Grid corner one cell outside the box, cell counts covering box + 2 cells."""
    gmin = tuple(f32(b - cell) for b in box_min)
    dims = tuple(int(math.ceil((hi - lo) / cell)) + 2 for lo, hi in zip(box_min, box_max))
    return gmin, dims


def lattice_mass(rho0: float, spacing: float, h: float) -> float:
    """Mass that gives a filled cubic lattice of this spacing exactly the rest
    density under the poly6 kernel (self included)."""
    R = int(math.ceil(h / spacing))
    acc = 0.0
    for k in range(-R, R + 1):
        for j in range(-R, R + 1):
            for i in range(-R, R + 1):
                r2 = (i * i + j * j + k * k) * spacing * spacing
                if r2 < h * h:
                    acc += (h * h - r2) ** 3
    return rho0 / (315.0 / (64.0 * math.pi * h ** 9) * acc)


def dam_break(
    nxyz: Sequence[int],
    spacing: float,
    box: Sequence[float],
    h: float,
    *,
    method: int = PCISPH,
    profile: int = PROFILE_CONFIG,
    dt: float = 1e-3,
    mass: Optional[float] = None,
    rho0: float = 1000.0,
    k: float = 3.0,
    mu: float = 0.01,
    eta: float = 0.01,
    min_iters: int = 3,
    max_iters: int = 50,
    jitter: float = 1e-4,
    seed: int = 0,
    steps: int = 0,
    name: str = "",
    nbr_cap: int = 128,
    skin: Optional[float] = None,
    xsph: Optional[float] = None,
) -> Scene:
    box_min = (0.0, 0.0, 0.0)
    box_max = tuple(float(b) for b in box)
    if skin is None:
        skin = 0.0
    if xsph is None:
        xsph = 0.25 if (profile == PROFILE_CONFIG and method == PCISPH) else 0.0
    cell = cell_for(h * (1.0 + skin), exact_reference=(profile == PROFILE_REF))
    gmin, dims = grid_for(box_min, box_max, cell)
    n = int(nxyz[0]) * int(nxyz[1]) * int(nxyz[2])
    m = lattice_mass(rho0, spacing, h) if mass is None else mass
    wk = 0.5 / (dt * dt)
    return Scene(
        n=n, box_min=box_min, box_max=box_max, grid_min=gmin, cell=cell, dims=dims, h=h, mass=m,
        rho0=rho0, k=k, mu=mu, sigma=0.0 if profile == PROFILE_CONFIG else 0.0728, l=7.065,
        particle_radius=f32(spacing / 2), dt=f32(dt), method=method, profile=profile,
        min_iters=min_iters, max_iters=max_iters, eta=eta, wall_k=wk, wall_c=math.sqrt(wk),
        blocks=[Block(tuple(int(v) for v in nxyz), spacing, (0.0, 0.0, 0.0), jitter, seed)],
        name=name, steps=steps, nbr_cap=nbr_cap, spacing=spacing, skin=skin, xsph=xsph,
    )


def dashpot_from_restitution(k_n: float, mass: float, restitution: float) -> float:
    """Normal dashpot c_n of a linear spring-dashpot contact between two
    equal spheres of this mass that gives the coefficient of restitution e:
    c_n = 2 zeta sqrt(k_n m_eff), m_eff = m/2, zeta = -ln e / sqrt(pi^2 + ln^2 e)
    (the damped oscillator's half-period rebound)."""
    le = math.log(restitution)
    zeta = -le / math.sqrt(math.pi ** 2 + le ** 2)
    return 2.0 * zeta * math.sqrt(k_n * mass / 2.0)


def dem_block(
    nxyz: Sequence[int],
    spacing: float,
    origin: Sequence[float],
    box: Sequence[float],
    radius: float,
    *,
    profile: int = PROFILE_CONFIG,
    density: float = 2500.0,
    k_n: float = 1e4,
    restitution: float = 0.3,
    spring: float = 0.0,
    damping: float = 0.0,
    shear: float = 0.0,
    attraction: float = 0.0,
    h: Optional[float] = None,
    dt: float = 1e-4,
    jitter: float = 1e-4,
    seed: int = 0,
    name: str = "",
) -> Scene:
    """A lattice block of DEM spheres (PSB_DEM) in a box [0, box].

    Config profile: linear spring-dashpot with k_n and the dashpot for the
    given restitution; the lists hold every pair within h = 2 radius.
    Reference profile: collideParticle's spring, damping, shear and
    attraction, over lists of radius h (the interaction radius)."""
    box_min = (0.0, 0.0, 0.0)
    box_max = tuple(float(b) for b in box)
    m = 4.0 / 3.0 * math.pi * radius ** 3 * density
    if h is None:
        h = 2.0 * radius
    cell = cell_for(h, exact_reference=(profile == PROFILE_REF))
    gmin, dims = grid_for(box_min, box_max, cell)
    if profile == PROFILE_CONFIG:
        spring, damping = k_n, dashpot_from_restitution(k_n, m, restitution)
    n = int(nxyz[0]) * int(nxyz[1]) * int(nxyz[2])
    return Scene(
        n=n, box_min=box_min, box_max=box_max, grid_min=gmin, cell=cell, dims=dims, h=h, mass=m,
        rho0=density, k=0.0, mu=0.0, sigma=0.0, l=0.0, particle_radius=f32(radius), dt=f32(dt), method=DEM,
        profile=profile, min_iters=0, max_iters=0, eta=0.0, wall_k=0.0, wall_c=0.0,
        blocks=[Block(tuple(int(v) for v in nxyz), spacing, tuple(float(o) for o in origin), jitter, seed)],
        name=name, steps=0, nbr_cap=64, spacing=spacing, dem_spring=spring, dem_damping=damping,
        dem_shear=shear, dem_attraction=attraction,
    )


# The synthetic scenes of the benchmark configurations (sizes from the scene text).
def config_scene(name: str) -> Scene:
    if name == "C0":   # plain WCSPH, 16,384 particles
        return dam_break((32, 32, 16), 0.01, (1.0, 0.5, 0.5), 0.02, method=WCSPH, dt=5e-4, mass=1e-3,
                         seed=0, steps=200, name="C0 WCSPH dam break 16,384")
    if name == "C1":   # PCISPH, 262,144 fluid particles (DEM spheres are a separate set)
        return dam_break((64, 64, 64), 0.01, (2.0, 1.0, 1.0), 0.02, dt=1e-3, mass=1e-3, seed=1, steps=500,
                         name="C1 PCISPH dam break 262,144")
    if name == "C2":   # PCISPH, 1,048,576 particles
        return dam_break((128, 128, 64), 0.005, (4.0, 2.0, 1.0), 0.01, dt=5e-4, seed=2, steps=1000,
                         name="C2 PCISPH dam break 1,048,576")
    if name == "C4":   # large PCISPH, 4,194,304 particles (obstacle not included here)
        return dam_break((256, 128, 128), 0.004, (3.0, 1.5, 1.0), 0.008, dt=5e-4, eta=0.005, seed=4, steps=300,
                         name="C4 PCISPH dam break 4,194,304")
    raise ValueError(f"unknown scene {name!r}")


def batch_scenes(n_scenes: int = 64, seed: int = 3, n_range=(4096, 131072), spacing: float = 0.01, h: float = 0.02,
                 side=(1.0, 2.0), fill=(0.4, 0.7), dt: float = 5e-4, warm_start: int = WARM_LEARNED,
                 jitter: float = 1e-4, steps: int = 300) -> List[Scene]:
    """Independent PCISPH dam breaks for one batch (config C3): particle
    counts log-uniform in n_range, each a lattice block at `spacing` in the
    corner of its own box, its height `fill` of the box's, box sides uniform
    in `side`; all drawn from `seed`. The block's footprint is square,
    nx = nz = round(sqrt(N / ny)), so the count is N up to that rounding.
    The scenes share every constant but their boxes and counts (a batch's
    requirement); each has its own jitter seed."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n_scenes):
        target = math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))
        box = tuple(float(round(v, 3)) for v in rng.uniform(side[0], side[1], 3))
        f = rng.uniform(fill[0], fill[1])
        ny = max(2, int(round(f * box[1] / spacing)))
        nxz = max(2, int(round(math.sqrt(target / ny))))
        nxz = min(nxz, int(box[0] / spacing) - 2, int(box[2] / spacing) - 2)
        sc = dam_break((nxz, ny, nxz), spacing, box, h, dt=dt, seed=seed * 1000 + s, jitter=jitter, steps=steps,
                       name=f"C3 scene {s}")
        out.append(sc.replace(warm_start=warm_start))
    return out


def c1_scenes(fluid_n=(64, 64, 64), dem_n=(16, 16, 16), seed: int = 1):
    """Config C1: the 262,144-particle PCISPH dam break (2 x 1 x 1 m box,
    dt = 1e-3) and 4,096 DEM spheres (radius 0.01 m, density 2500 kg/m^3,
    k_n = 1e4 N/m, restitution 0.3) on a 16^3 lattice of spacing 0.021 m
    above the fluid block, same box and time step. Returns (fluid, spheres);
    smaller counts give the same set-up at test size."""
    fluid = dam_break(fluid_n, 0.01, (2.0, 1.0, 1.0), 0.02, dt=1e-3, mass=1e-3, seed=seed, steps=500,
                      name="C1 PCISPH dam break %d" % (fluid_n[0] * fluid_n[1] * fluid_n[2]))
    top = fluid_n[1] * 0.01
    spheres = dem_block(dem_n, 0.021, (0.1, top + 0.02, 0.1), (2.0, 1.0, 1.0), 0.01, density=2500.0, k_n=1e4,
                        restitution=0.3, dt=1e-3, seed=seed + 100, name="C1 DEM spheres")
    return fluid, spheres


def sphere_shell(centre, radius: float, spacing: float, layers: int = 2) -> np.ndarray:
    """Boundary particles of a solid sphere: the points of the cubic lattice
    of this spacing (aligned on the centre) whose distance to the centre lies
    in [radius - layers spacing, radius). A shell of two spacings covers the
    kernel's reach h = 2 spacing from outside."""
    c = np.asarray(centre, np.float64)
    m = int(math.ceil(radius / spacing)) + 1
    ax = np.arange(-m, m + 1) * spacing
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    d = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    sel = (d < radius) & (d >= radius - layers * spacing)
    return (np.stack([X[sel], Y[sel], Z[sel]], 1) + c).astype(np.float32)


def ref_scene(nxyz=(12, 10, 8), spacing=0.01, box=(0.3, 0.3, 0.3), h=0.02, method=PCISPH, dt=5e-4,
              seed=7, jitter=1e-4) -> Scene:
    """Small scene in the reference-compatible profile (parity tests)."""
    s = dam_break(nxyz, spacing, box, h, method=method, profile=PROFILE_REF, dt=dt, mass=1e-3, seed=seed,
                  jitter=jitter, name="ref-profile scene")
    return s
