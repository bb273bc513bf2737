"""Seeded scene construction: the host-side mirror of the reference's scene setup.

Mirrors, with a seeded PRNG instead of std::rand(time(NULL)):
  - Simulation::GenerateParticleCube (Simulation.cpp:599-662): lattice blocks, x outer,
    z inner loop order;
  - Simulation::InitializeBoundaryParticles (Simulation.cpp:425-556): the one-particle
    thick box (floor at y = -r, walls just outside x,z = +-1), evaluated in float32;
  - ParticleSet::AppendExtraMemory (Particle.cpp:404-429): each set padded to
    full = n_water + n_snow with INF positions;
  - ParticleSystem::SetupCUDAMemory (ParticleSystem.cpp:148-858): initial contrib,
    predicate, trackId (1..N), iter_end[i] = maxc*i and empty interlink records.

Buffers the reference leaves uninitialised get a defined value here: cell_start is
all-empty, cell_end 0, grid_index the identity, contrib 1 in the padding.
"""
import functools
import math
from dataclasses import dataclass, field

import numpy as np

from .abi import PARTICLE_FIELDS, DEFAULT_FLAGS
from .params import make_sim_params

UMAX = np.uint32(0xFFFFFFFF)


def _alloc_set(full, maxc, dtype=np.float32):
    s = {}
    for name, kind in PARTICLE_FIELDS:
        if kind == "v3":
            s[name] = np.zeros((full, 3), dtype)
        elif kind == "f":
            s[name] = np.zeros(full, dtype)
        elif kind == "u":
            s[name] = np.zeros(full, np.uint32)
        elif kind == "u1":
            s[name] = np.zeros(1, np.uint32)
        elif kind == "urec":
            s[name] = np.full(full * maxc, UMAX, np.uint32)
        elif kind == "frec":
            s[name] = np.zeros(full * maxc, dtype)
    return s


def _alloc_cells(n_entries, num_cells, dtype=np.float32):
    return dict(
        grid_hash=np.zeros(n_entries, np.uint32),
        grid_index=np.arange(n_entries, dtype=np.uint32),
        cell_start=np.full(num_cells, UMAX, np.uint32),
        cell_end=np.zeros(num_cells, np.uint32),
        sorted_pos=np.zeros((n_entries, 3), dtype),
    )


@dataclass
class HostWorld:
    """Complete solver state in host memory, laid out like the reference's device buffers."""
    params: object
    sph: dict
    dem: dict
    bnd: dict
    buffer: dict
    sph_cd: dict
    dem_cd: dict
    b_cd: dict
    n_sph: int
    n_dem: int
    n_b: int
    full: int
    maxc: int
    scene: list                     # fluid_start_time, solid_start_time, current_time
    dt: float = 1.0 / 240.0
    iterations: int = 3
    substeps_per_frame: int = 4
    flags: dict = field(default_factory=lambda: dict(DEFAULT_FLAGS))
    temperature_variation: float = 0.0
    name: str = ""
    init_links: bool = False
    domain: tuple = (-1.0, 1.0, -1.0, 1.0, 0.0)   # walls x_min, x_max, z_min, z_max and floor y

    def copy(self):
        def cp(d):
            return {k: v.copy() for k, v in d.items()}
        return HostWorld(self.params, cp(self.sph), cp(self.dem), cp(self.bnd), cp(self.buffer),
                         cp(self.sph_cd), cp(self.dem_cd), cp(self.b_cd), self.n_sph, self.n_dem,
                         self.n_b, self.full, self.maxc, list(self.scene), self.dt, self.iterations,
                         self.substeps_per_frame, dict(self.flags), self.temperature_variation,
                         self.name, self.init_links, tuple(self.domain))


def lattice(counts, spacing, origin_min, jitter=0.0, rng=None):
    """Particles on a lattice, loop order x (outer), y, z (inner) as GenerateParticleCube."""
    nx, ny, nz = counts
    s = np.float32(spacing)
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    pos = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(np.float32) * s
    pos += np.asarray(origin_min, np.float32)
    if jitter:
        pos += rng.uniform(-jitter, jitter, size=pos.shape).astype(np.float32)
    return pos.astype(np.float32)


def boundary_box(particle_radius, half_x=1.0, half_y=1.0, half_z=1.0):
    """InitializeBoundaryParticles (Simulation.cpp:425-556) in float32 arithmetic.  The
    half extents are the reference's 1 m unless a wider domain asks for more."""
    return _boundary_box(float(np.float32(particle_radius)), float(half_x), float(half_y), float(half_z)).copy()


@functools.lru_cache(maxsize=4)
def _boundary_box(particle_radius, half_x, half_y, half_z):
    f = np.float32
    thickness = 1
    d = f(2.0) * f(particle_radius)
    pts = []
    he1 = (f(half_x), d * f(thickness) / f(2.0), f(half_z))
    nx, nz = int(he1[0] / d), int(he1[2] / d)
    bo_y = f(-0.5) * d
    left, right = np.inf, -np.inf
    for i in range(-nx - thickness, nx + thickness):
        for j in range(0, thickness):
            for k in range(-nz - thickness, nz + thickness):
                x = f(0) + d * f(i)
                y = bo_y - d * f(j)
                z = f(0) + d * f(k)
                pts.append((x, y, z))
                left = min(left, x)
                right = max(right, x)
    left = f(left) - d
    right = f(right) + d
    he2 = (d * f(thickness) / f(2.0), f(half_y), f(half_z))
    ny, nz = int(he2[1] / d), int(he2[2] / d)
    lo = (left, f(ny) * d, f(0))
    ro = (right, f(ny) * d, f(0))
    back, front = np.inf, -np.inf
    for i in range(0, thickness):
        for j in range(-ny - thickness, ny):
            for k in range(-nz - thickness, nz + thickness):
                x = -d * f(i)
                y = d * f(j)
                z = d * f(k)
                pts.append((x + lo[0], y + lo[1], z + lo[2]))
                x = d * f(i)
                p = (x + ro[0], y + ro[1], z + ro[2])
                pts.append(p)
                back = min(back, p[2])
                front = max(front, p[2])
    back = f(back) - d
    front = f(front) + d
    he3 = (f(half_x), f(half_y), d * f(thickness) / f(2.0))
    nx, ny = int(he3[0] / d), int(he3[1] / d)
    bko = (f(0), f(ny) * d, back)
    fro = (f(0), f(ny) * d, front)
    for i in range(-nx - 2 * thickness, nx + 2 * thickness):
        for j in range(-ny - thickness, ny):
            for k in range(0, thickness):
                x = d * f(i)
                y = d * f(j)
                z = -d * f(k)
                pts.append((x + bko[0], y + bko[1], z + bko[2]))
                z = d * f(k)
                pts.append((x + fro[0], y + fro[1], z + fro[2]))
    return np.asarray(pts, np.float32)


def build_world(water_pos, snow_pos, T_water, T_snow, params=None, mass=None, boundary=None,
                name="", **kw):
    """Assemble a HostWorld from particle positions, as SetupCUDAMemory initialises it."""
    p = params if params is not None else make_sim_params()
    maxc = int(p.maximum_connection)
    n_sph, n_dem = len(water_pos), len(snow_pos)
    full = n_sph + n_dem
    if mass is None:
        mass = float(p.rest_density) * (2.0 * float(p.particle_radius)) ** 3
    m = np.float32(mass)
    inv = np.float32(1.0) / m
    bpos = boundary_box(p.particle_radius) if boundary is None else np.asarray(boundary, np.float32)
    n_b = len(bpos)

    def fill(s, pos, n, T, id0):
        s["positions"][:] = np.inf
        s["positions"][:n] = pos
        s["predict_positions"][:] = s["positions"]
        s["new_positions"][:] = s["positions"]
        s["mass"][:] = m
        s["massInv"][:] = inv
        s["T"][:n] = T
        s["new_T"][:] = s["T"]
        s["contrib"][:] = 1.0
        s["mass_scale"][:] = 1.0
        s["predicate"][:n] = 1
        s["new_end"][0] = n
        s["iter_end"][:] = np.arange(full, dtype=np.uint32) * np.uint32(maxc)
        s["trackId"][:n] = np.arange(id0, id0 + n, dtype=np.uint32)

    sph = _alloc_set(full, maxc)
    dem = _alloc_set(full, maxc)
    fill(sph, water_pos, n_sph, T_water, 1)
    fill(dem, snow_pos, n_dem, T_snow, 1 + n_sph)
    bnd = _alloc_set(n_b, maxc)
    bnd["positions"][:] = bpos
    bnd["predict_positions"][:] = bpos
    bnd["new_positions"][:] = bpos
    bnd["mass"][:] = m
    bnd["massInv"][:] = inv
    bnd["contrib"][:] = 1.0
    bnd["mass_scale"][:] = 1.0
    bnd["iter_end"][:] = np.arange(n_b, dtype=np.uint32) * np.uint32(maxc)
    buffer = _alloc_set(full, maxc)
    nc = int(p.num_cells)
    w = HostWorld(p, sph, dem, bnd, buffer, _alloc_cells(full, nc), _alloc_cells(full, nc),
                  _alloc_cells(n_b, nc), n_sph, n_dem, n_b, full, maxc, [0.0, 0.0, 0.0],
                  name=name, **kw)
    return w


# ----------------------------------------------------------------- named scenes
def _block(counts, spacing, centre_xz, bottom_y, jitter, rng):
    nx, ny, nz = counts
    s = float(np.float32(spacing))
    origin = (centre_xz[0] - 0.5 * s * (nx - 1), bottom_y, centre_xz[1] - 0.5 * s * (nz - 1))
    return lattice(counts, spacing, origin, jitter, rng)


def scene_drop(water_counts, snow_counts, *, seed=0, spacing=0.02, water_jitter=0.0,
               snow_jitter=0.0, drop_height=0.3, T_water=100.0, T_snow=-10.0, name="",
               params=None, **kw):
    """A water block dropped onto a snow block resting on the floor (centred at x = z = 0)."""
    rng = np.random.default_rng(seed)
    p = params if params is not None else make_sim_params()
    r = float(p.particle_radius)
    snow = _block(snow_counts, spacing, (0.0, 0.0), r, snow_jitter, rng)
    snow_top = r + spacing * (snow_counts[1] - 1)
    water = _block(water_counts, spacing, (0.0, 0.0), snow_top + drop_height, water_jitter, rng)
    return build_world(water, snow, T_water, T_snow, params=p, name=name, **kw)


def config0(seed=0):
    """1,000 water (10^3, jitter +-2 mm, 100 C) dropped 0.3 m onto a 16^3 snow block (-10 C)."""
    return scene_drop((10, 10, 10), (16, 16, 16), seed=seed, water_jitter=0.002,
                      name="config0: 1000 water + 4096 snow")


def config1(seed=0):
    """5,888 water (8x92x8 column, 100 C) above 147,928 snow (82x22x82 box, jitter +-2 mm, -10 C)."""
    return scene_drop((8, 92, 8), (82, 22, 82), seed=seed, snow_jitter=0.002, drop_height=0.1,
                      name="config1: 5888 water + 147928 snow", init_links=True)


def tiny(seed=0, water=(4, 4, 4), snow=(6, 4, 6), drop=0.06, **kw):
    """A small scene that the FP32/FP64 oracle steps through in well under a second."""
    return scene_drop(water, snow, seed=seed, water_jitter=0.002, snow_jitter=0.002,
                      drop_height=drop, name="tiny", **kw)


def config2(seed=0, n_scenes=64, lo=2000, hi=40000):
    """Scenes for a batched run: particle counts log-uniform in [lo, hi] per scene, water
    fraction uniform in 0.02-0.3, drop height uniform in 0.1-0.5 m, snow temperature uniform
    in -20..-2 C (water 100 C); each block is the nearest cube lattice (spacing 0.02 m,
    jitter +-2 mm), snow resting on the floor with initial interlinks.  Returns a list of
    HostWorlds sharing one SimParams."""
    rng = np.random.default_rng(seed)
    p = make_sim_params()
    worlds = []
    for s in range(n_scenes):
        n = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        frac = rng.uniform(0.02, 0.3)
        drop = rng.uniform(0.1, 0.5)
        t_snow = rng.uniform(-20.0, -2.0)
        kw = max(1, int(round((n * frac) ** (1.0 / 3.0))))
        ks = max(1, int(round((n * (1.0 - frac)) ** (1.0 / 3.0))))
        worlds.append(scene_drop((kw, kw, kw), (ks, ks, ks), seed=seed * 1000 + s, water_jitter=0.002,
                                 snow_jitter=0.002, drop_height=drop, T_snow=float(np.float32(t_snow)),
                                 params=p, name="config2 scene %d" % s, init_links=True))
    return worlds


def config3(seed=0):
    """Adjoint scene: 1,024 water (8x16x8 column, jitter +-2 mm, 100 C) falling onto an
    8,192-particle snow block (32x8x32, jitter +-2 mm, -10 C) with initial interlinks.
    Phase change is off: the adjoint holds phase flags fixed, so a differentiated run may
    not move particles between sets."""
    w = scene_drop((8, 16, 8), (32, 8, 32), seed=seed, water_jitter=0.002, snow_jitter=0.002, drop_height=0.1,
                   name="config3: 1024 water + 8192 snow", init_links=True)
    w.flags["change_phase"] = False
    return w


def config4(seed=0):
    """The large scene: a 1,048,576-particle snow block (128 x 64 x 128, jitter +-2 mm, -10 C)
    with initial interlinks, and 131,072 water particles (100 C) in 8 columns of 16,384
    (16 x 64 x 16) dropped 0.3 m onto it.  It does not fit the reference's 2 m box, so the
    walls move to x, z = +-1.5 m (boundary box of the same construction, 3 m tall) and the
    grid grows to 128^3 cells of h (5.12 m per axis, wrapped)."""
    rng = np.random.default_rng(seed)
    p = make_sim_params(grid_size=(128, 128, 128))
    r, s = float(p.particle_radius), 0.02
    snow = _block((128, 64, 128), s, (0.0, 0.0), r, 0.002, rng)
    top = r + s * 63
    water = []
    for k in range(8):
        cx = -0.96 + 0.64 * (k % 4)
        cz = -0.48 + 0.96 * (k // 4)
        water.append(_block((16, 64, 16), s, (cx, cz), top + 0.3, 0.002, rng))
    water = np.concatenate(water)
    half = 1.5
    return build_world(water, snow, 100.0, -10.0, params=p, boundary=boundary_box(r, half, half, half),
                       name="config4: 131072 water + 1048576 snow", init_links=True,
                       domain=(-half, half, -half, half, 0.0))


def adjoint_tiny(seed=0):
    """A small scene for adjoint tests: 27 water particles dropped onto a 6x3x6 snow block
    with interlinks, phase change off."""
    w = scene_drop((3, 3, 3), (6, 3, 6), seed=seed, water_jitter=0.002, snow_jitter=0.002, drop_height=0.005,
                   name="adjoint tiny", init_links=True)
    w.flags["change_phase"] = False
    return w


SCENES = {"config0": config0, "config1": config1, "config3": config3, "config4": config4, "tiny": tiny}
