"""Solver constants: the host-side mirror of Simulation::SetupSimParams (Simulation.cpp:339-423).

The reference derives radius and support from a particle mass and a kernel
particle count; the benchmark scenes fix them instead (particle radius 0.01 m,
support h = 0.04 m, lattice spacing 0.02 m).  The particle mass defaults to
rest_density * spacing**3 = 0.008 kg so a rest lattice sits at the rest density.
Every other field takes the value SetupSimParams assigns, and the kernel
constants are evaluated with the same expressions (float pow, double pi).
"""
import math

import numpy as np

from .abi import SimParams


def _f32(x):
    return float(np.float32(x))


def poly6_w_fp64(distance, h):
    """SPHKernel::Poly6_W (SPHKernel.h:9-29): FP64 poly6 with support d <= h."""
    if 0.0 <= distance <= h:
        h = float(np.float32(h))
        d = float(np.float32(distance))
        q = h * h - d * d
        return _f32((315.0 / (64.0 * math.pi * h ** 9)) * q * q * q)
    return 0.0


def make_sim_params(particle_radius=0.01, effective_radius=0.04, rest_density=1000.0,
                    k_water=600.0, k_snow=2500.0, grid_size=(64, 64, 64),
                    maximum_connection=25, cell_size=None, world_origin=(0.0, 0.0, 0.0),
                    **overrides):
    """Build a SimParams struct; keyword overrides replace any named field."""
    p = SimParams()
    h = np.float32(effective_radius)
    r = np.float32(particle_radius)
    p.gravity[:] = (0.0, -9.8, 0.0)
    p.global_damping = 1.0
    p.maximum_speed = 10.0
    p.minimum_speed = 0.0
    p.particle_radius = r
    p.effective_radius = h
    p.rest_density = rest_density
    p.epsilon = 100.0
    p.pbd_epsilon = _f32(np.float32(0.01) * r)
    p.kernel_epsilon = _f32(np.float32(0.01) * h)
    gs = tuple(int(g) for g in grid_size)
    for g in gs:
        if g <= 0 or g & (g - 1):
            raise ValueError("grid sizes must be powers of two (the hash wraps with a mask)")
    p.grid_size[:] = gs
    p.num_cells = gs[0] * gs[1] * gs[2]
    p.world_origin[:] = world_origin
    cs = (h, h, h) if cell_size is None else cell_size
    p.cell_size[:] = cs
    p.boundary_damping = 0.15
    p.static_friction = 0.5
    p.kinematic_friction = 0.35
    p.scorr_coeff = 0.0
    p.sor_coeff = 0.25
    p.sph_viscosity = 0.01
    p.dem_viscosity = 0.1
    p.k_stretch = 0.25
    p.C_snow = 2090.0
    p.C_water = 4182.0
    p.k_snow = k_snow
    p.k_water = k_water
    p.freezing_point = 0.0
    p.T_homogeneous = -30.0
    p.blending_speed = 0.01
    h9 = float(np.float32(h) ** np.float32(9))
    h6 = float(np.float32(h) ** np.float32(6))
    p.poly6 = _f32(315.0 / (64.0 * math.pi * h9))
    p.poly6_G = _f32(-945.0 / (32.0 * math.pi * h9))
    p.spiky = _f32(15.0 / (math.pi * h6))
    p.spiky_G = _f32(-45.0 / (math.pi * h6))
    p.viscosity_laplacian = _f32(45.0 / (math.pi * h6))
    p.scorr_divisor = poly6_w_fp64(0.3 * float(h), float(h))
    p.maximum_connection = maximum_connection
    p.k_refreezing = 0.75
    p.break_threshold = 1.05
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(k)
        cur = getattr(p, k)
        if hasattr(cur, "__len__"):
            cur[:] = v
        else:
            setattr(p, k, v)
    return p


def params_dict(p):
    out = {}
    for name, _ in SimParams._fields_:
        v = getattr(p, name)
        out[name] = list(v) if hasattr(v, "__len__") else v
    return out
