"""ctypes mirrors of the C-ABI structs declared in include/snow_b200.h.

The structs reproduce the reference's data model field for field:
ParticleDeviceData (Particle.h:14-52), CellData (NeighborSearch.h:19-26),
SimParams (SimParams.h:7-62) and SceneParams (SceneParams.h:4-9).
"""
import ctypes as C

# Field order of ParticleDeviceData (Particle.h:14-52).
PARTICLE_FIELDS = (
    ("positions", "v3"), ("predict_positions", "v3"), ("new_positions", "v3"),
    ("velocity", "v3"), ("force", "v3"), ("correction", "v3"),
    ("mass", "f"), ("massInv", "f"), ("density", "f"), ("C", "f"), ("lambda_", "f"),
    ("volume", "f"), ("T", "f"), ("new_T", "f"), ("contrib", "f"), ("mass_scale", "f"),
    ("predicate", "u"), ("scan_index", "u"), ("new_end", "u1"),
    ("connect_record", "urec"), ("iter_end", "u"), ("connect_length", "frec"),
    ("new_index", "u"), ("trackId", "u"),
)
CELL_FIELDS = ("grid_hash", "grid_index", "cell_start", "cell_end", "sorted_pos")


class ParticleDeviceData(C.Structure):
    _fields_ = [(name, C.c_void_p) for name, _ in PARTICLE_FIELDS]


class CellData(C.Structure):
    _fields_ = [(name, C.c_void_p) for name in CELL_FIELDS]


class SimParams(C.Structure):
    _fields_ = [
        ("gravity", C.c_float * 3),
        ("global_damping", C.c_float), ("maximum_speed", C.c_float), ("minimum_speed", C.c_float),
        ("epsilon", C.c_float), ("pbd_epsilon", C.c_float), ("kernel_epsilon", C.c_float),
        ("effective_radius", C.c_float), ("particle_radius", C.c_float),
        ("rest_density", C.c_float), ("scorr_coeff", C.c_float), ("scorr_divisor", C.c_float),
        ("boundary_damping", C.c_float), ("static_friction", C.c_float), ("kinematic_friction", C.c_float),
        ("k_stretch", C.c_float),
        ("k_water", C.c_float), ("k_snow", C.c_float), ("C_water", C.c_float), ("C_snow", C.c_float),
        ("freezing_point", C.c_float),
        ("blending_speed", C.c_float),
        ("sor_coeff", C.c_float), ("sph_viscosity", C.c_float), ("dem_viscosity", C.c_float),
        ("world_origin", C.c_float * 3), ("cell_size", C.c_float * 3),
        ("grid_size", C.c_uint32 * 3), ("num_cells", C.c_uint32),
        ("poly6", C.c_float), ("poly6_G", C.c_float), ("spiky", C.c_float), ("spiky_G", C.c_float),
        ("viscosity_laplacian", C.c_float),
        ("maximum_connection", C.c_uint32),
        ("T_homogeneous", C.c_float), ("k_refreezing", C.c_float), ("break_threshold", C.c_float),
    ]


class Batch(C.Structure):
    """snowb_batch: scene layout of a batched run and the scene-id array of each set."""
    _fields_ = [("scenes_x", C.c_uint32), ("scenes_z", C.c_uint32), ("scene_sph", C.c_void_p),
                ("scene_dem", C.c_void_p), ("scene_boundary", C.c_void_p), ("scene_buffer", C.c_void_p)]


class SceneParams(C.Structure):
    _fields_ = [("fluid_start_time", C.c_float), ("solid_start_time", C.c_float),
                ("current_time", C.c_float)]


# Boolean flags of snow_simulation() (cuda_simulation.cuh:52-75), in argument order.
FLAG_NAMES = (
    "sph_dem_correction", "sph_sph_correction", "dem_friction", "compute_temperature",
    "change_phase", "simulate_freezing", "simulate_melting", "dem_viscosity",
    "use_interlink", "dynamic_max_connections", "cd_on",
)

# Defaults of Simulation::StepCUDA's ImGui toggles (Simulation.cpp:181-193).
DEFAULT_FLAGS = dict(
    sph_dem_correction=True, sph_sph_correction=False, dem_friction=True,
    compute_temperature=True, change_phase=True, simulate_freezing=True,
    simulate_melting=True, dem_viscosity=True, use_interlink=True,
    dynamic_max_connections=False, cd_on=True,
)


def flag_bits(flags):
    """Pack the flag dict into the bitfield used by the oracle (bit i = FLAG_NAMES[i])."""
    bits = 0
    for i, name in enumerate(FLAG_NAMES):
        if flags.get(name, False):
            bits |= 1 << i
    return bits


QUIRKS_REFERENCE = 0
QUIRKS_FIXED = 1


def _header_limit(name):
    """Value of a `#define NAME (1u << k)` limit in include/snow_b200.h."""
    import os
    import re
    here = os.path.dirname(os.path.abspath(__file__))
    txt = open(os.path.join(here, "..", "include", "snow_b200.h")).read()
    m = re.search(r"#define\s+%s\s+\(1u\s*<<\s*(\d+)\)" % name, txt)
    if not m:
        raise RuntimeError("%s not found in include/snow_b200.h" % name)
    return 1 << int(m.group(1))


# Limits of snowb_sort_particles_static (its static device scratch), from the header.
STATIC_SORT_MAX_PARTICLES = _header_limit("SNOWB_STATIC_SORT_MAX_PARTICLES")
STATIC_SORT_MAX_CELLS = _header_limit("SNOWB_STATIC_SORT_MAX_CELLS")
