"""Loader for libsnowb200.so (the CUDA library) with ctypes signatures of include/snow_b200.h.

There is no fallback: if the library is missing or fails to load, import of the solver
raises, so nothing silently runs on another path.
"""
import ctypes as C
import os

from .abi import ParticleDeviceData, CellData, SimParams, SceneParams, Batch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsnowb200.so")


class AdjointIO(C.Structure):
    """snowb_adjoint_io: device gradient buffers (in/out) and the accumulated parameter gradients."""
    _fields_ = [("gx_sph", C.c_void_p), ("gv_sph", C.c_void_p), ("gT_sph", C.c_void_p),
                ("gx_dem", C.c_void_p), ("gv_dem", C.c_void_p), ("gT_dem", C.c_void_p),
                ("gL_dem", C.c_void_p), ("grad_params", C.c_double * 4)]


class StepOptions(C.Structure):
    _fields_ = [("quirks", C.c_int), ("substeps", C.c_int), ("stop_after", C.c_int),
                ("use_graph", C.c_int), ("sync", C.c_int)]


# Every symbol declared in include/snow_b200.h.
EXPORTS = (
    "snowb_allocate_array", "snowb_set_sim_params", "snowb_compute_grid_size", "snowb_calculate_hash",
    "snowb_sort_particles", "snowb_reorder_data", "snowb_compute_boundary_volume", "snowb_integrate_pbd",
    "snowb_connect_and_record", "snowb_snow_simulation", "snowb_snow_simulation_ex", "snowb_read_sizes",
    "snowb_set_quirks", "snowb_set_stream", "snowb_synchronize", "snowb_energy_momentum", "snowb_release",
    "snowb_last_error", "snowb_last_error_string", "snowb_launch_count", "snowb_profile_begin",
    "snowb_profile_end", "snowb_profile_timeline", "snowb_device_counters",
    "snowb_sort_particles_static",
    "snowb_batch_num_cells", "snowb_batch_calculate_hash", "snowb_batch_sort_particles",
    "snowb_batch_reorder_data", "snowb_batch_compute_boundary_volume", "snowb_batch_connect_and_record",
    "snowb_batch_snow_simulation",
    "snowb_adjoint_begin", "snowb_adjoint_end", "snowb_adjoint_backward", "snowb_adjoint_release",
    "snowb_autotune", "snowb_autotune_table", "snowb_autotune_load", "snowb_autotune_reset",
    "snowb_set_domain",
    "snowb_export_bgeo", "snowb_export_bgeo_async", "snowb_export_wait", "snowb_write_bgeo_host",
    "snowb_render_clear", "snowb_render_points", "snowb_render_clear_colour",
    "snowb_ssfr_workspace_bytes", "snowb_render_fluid", "snowb_ssfr_clear", "snowb_ssfr_sphere_depth",
    "snowb_ssfr_thickness", "snowb_ssfr_smooth", "snowb_ssfr_compose", "snowb_ssfr_matrices",
)

_lib = None


class SnowError(RuntimeError):
    pass


def load(path=LIB_PATH):
    """Load the CUDA library once; raise if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise SnowError("libsnowb200.so not built (run snowsimulation_b200/build.py): %s" % path)
    lib = C.CDLL(path)
    PD, PPD, CD = ParticleDeviceData, C.POINTER(ParticleDeviceData), CellData
    u32, pu32, i, f = C.c_uint32, C.POINTER(C.c_uint32), C.c_int, C.c_float
    sig = {
        "snowb_allocate_array": [C.POINTER(C.c_void_p), C.c_size_t],
        "snowb_set_sim_params": [C.POINTER(SimParams)],
        "snowb_compute_grid_size": [u32, u32, pu32, pu32],
        "snowb_calculate_hash": [CD, C.c_void_p, u32],
        "snowb_sort_particles": [CD, u32],
        "snowb_reorder_data": [CD, C.c_void_p, u32, u32],
        "snowb_compute_boundary_volume": [CD, C.c_void_p, C.c_void_p, u32],
        "snowb_integrate_pbd": [PPD, f, u32, i],
        "snowb_connect_and_record": [PPD, u32, CD, i],
        "snowb_snow_simulation": [PPD, pu32, PPD, pu32, PPD, u32, u32, PPD, CD, CD, CD,
                                  C.POINTER(SceneParams), f, i] + [i] * 11 + [f],
        "snowb_read_sizes": [pu32, pu32],
        "snowb_set_quirks": [i],
        "snowb_set_stream": [C.c_void_p],
        "snowb_synchronize": [],
        "snowb_energy_momentum": [PPD, u32, PPD, u32, C.POINTER(C.c_double)],
        "snowb_release": [],
        "snowb_last_error": [],
        "snowb_launch_count": [C.POINTER(C.c_uint64)],
        "snowb_profile_begin": [],
        "snowb_profile_end": [C.c_char_p, C.c_size_t],
        "snowb_profile_timeline": [C.c_char_p, C.c_size_t],
        "snowb_device_counters": [C.POINTER(C.c_uint32), C.c_int],
        "snowb_sort_particles_static": [CD, u32],
    }
    sig["snowb_snow_simulation_ex"] = sig["snowb_snow_simulation"] + [C.POINTER(StepOptions)]
    PB = C.POINTER(Batch)
    sig.update({
        "snowb_batch_num_cells": [PB, pu32],
        "snowb_batch_calculate_hash": [PB, CD, C.c_void_p, C.c_void_p, u32],
        "snowb_batch_sort_particles": [PB, CD, u32],
        "snowb_batch_reorder_data": [PB, CD, C.c_void_p, u32],
        "snowb_batch_compute_boundary_volume": [PB, CD, C.c_void_p, C.c_void_p, u32],
        "snowb_batch_connect_and_record": [PB, PPD, u32, CD, i],
        "snowb_batch_snow_simulation": [PB] + sig["snowb_snow_simulation_ex"],
        "snowb_adjoint_begin": [],
        "snowb_adjoint_end": [pu32],
        "snowb_adjoint_backward": [C.POINTER(AdjointIO)],
        "snowb_adjoint_release": [],
        "snowb_autotune": sig["snowb_snow_simulation"] + [i, i, PB],
        "snowb_autotune_table": [C.c_char_p, C.c_size_t],
        "snowb_autotune_load": [C.c_char_p],
        "snowb_autotune_reset": [],
        "snowb_set_domain": [f, f, f, f, f],
        "snowb_export_bgeo": [PPD, u32, C.c_char_p, C.POINTER(C.c_float), f, i, i],
        "snowb_export_bgeo_async": [PPD, u32, C.c_char_p, C.POINTER(C.c_float), f, i, i],
        "snowb_export_wait": [],
        "snowb_write_bgeo_host": [C.c_void_p, u32, C.c_char_p, C.POINTER(C.c_float), f, i, i],
        # camera and colour structs (render.py) are passed by address
        "snowb_render_clear": [C.c_void_p, C.c_void_p, C.c_void_p],
        "snowb_render_points": [PPD, u32, C.c_void_p, C.c_void_p, u32, C.c_void_p, C.c_void_p],
        "snowb_render_clear_colour": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
        "snowb_ssfr_workspace_bytes": [C.c_void_p, C.POINTER(C.c_uint64)],
        "snowb_render_fluid": [PPD, u32, PPD, u32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
        "snowb_ssfr_clear": [C.c_void_p, C.c_void_p, C.c_void_p],
        "snowb_ssfr_sphere_depth": [PPD, u32, C.c_void_p, C.c_void_p, C.c_void_p],
        "snowb_ssfr_thickness": [PPD, u32, C.c_void_p, C.c_void_p],
        "snowb_ssfr_smooth": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
        "snowb_ssfr_compose": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
        "snowb_ssfr_matrices": [C.c_void_p, C.c_void_p],
    })
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_int
    lib.snowb_last_error_string.argtypes = []
    lib.snowb_last_error_string.restype = C.c_char_p
    _lib = lib
    return lib


def check(rc):
    if rc != 0:
        msg = _lib.snowb_last_error_string().decode() if _lib is not None else ""
        raise SnowError("libsnowb200 error %d: %s" % (rc, msg))
    return rc
