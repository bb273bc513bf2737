"""ctypes driver for the reference's own CUDA solver (TEST INFRASTRUCTURE).

oracle/_ref/libsnowref.so is the reference's cuda_simulation.cu compiled unchanged for
sm_100a with ref_harness.cu, with the project's fast math; libsnowref_ieee.so is the same
build with IEEE arithmetic and no contraction (both built by ref_build.sh from the
reference's sources).  RefWorld runs a HostWorld through it so tests can pin the CPU
oracle to the reference's actual results, and the reference arm of the benchmark times
it.  Only one RefWorld can exist at a time (the reference keeps its parameters in a
__constant__ symbol and static counters).
"""
import ctypes as C
import os

import numpy as np

from snowsimulation_b200.abi import PARTICLE_FIELDS, CELL_FIELDS, FLAG_NAMES, SimParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {"fast": os.path.join(HERE, "_ref", "libsnowref.so"),
        "ieee": os.path.join(HERE, "_ref", "libsnowref_ieee.so")}

_libs = {}


def available(variant="fast"):
    return os.path.exists(LIBS[variant])


def load(variant="fast"):
    if variant not in _libs:
        lib = C.CDLL(LIBS[variant])
        u32 = C.c_uint32
        lib.ref_create.argtypes = [C.POINTER(SimParams), u32, u32, u32, u32, u32]
        lib.ref_copy_set.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.c_int]
        lib.ref_copy_cells.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.c_int]
        lib.ref_init_boundary.argtypes = []
        lib.ref_init_links.argtypes = [C.c_int]
        lib.ref_step.argtypes = [C.POINTER(C.c_float), C.c_float, C.c_int, C.POINTER(C.c_int), C.c_float,
                                 C.POINTER(C.c_uint32)]
        lib.ref_step_until.argtypes = [C.POINTER(C.c_float), C.c_float, C.c_int, C.POINTER(C.c_int), C.c_float,
                                       C.c_int, C.POINTER(C.c_uint32)]
        lib.ref_destroy.argtypes = []
        _libs[variant] = lib
    return _libs[variant]


class RefWorld:
    def __init__(self, host_world, variant="fast"):
        self.lib = load(variant)
        w = host_world.copy()
        self.w = w
        self.params = w.params
        rc = self.lib.ref_create(C.byref(self.params), w.full, w.n_sph, w.n_dem, w.n_b, w.maxc)
        assert rc == 0, "ref_create failed (%d)" % rc
        for s, d in enumerate((w.sph, w.dem, w.bnd, w.buffer)):
            self._copy_set(s, d, True)
        for s, d in enumerate((w.sph_cd, w.dem_cd, w.b_cd)):
            self._copy_cells(s, d, True)

    def _copy_set(self, s, d, to_dev):
        ptrs = (C.c_void_p * 24)(*[d[n].ctypes.data for n, _ in PARTICLE_FIELDS])
        assert self.lib.ref_copy_set(s, ptrs, 1 if to_dev else 0) == 0

    def _copy_cells(self, s, d, to_dev):
        ptrs = (C.c_void_p * 5)(*[d[n].ctypes.data for n in CELL_FIELDS])
        assert self.lib.ref_copy_cells(s, ptrs, 1 if to_dev else 0) == 0

    def setup(self):
        assert self.lib.ref_init_boundary() == 0
        if self.w.init_links:
            assert self.lib.ref_init_links(int(bool(self.w.flags.get("dynamic_max_connections")))) == 0
        return self

    def step(self, stop_after=None):
        """snow_simulation itself, or (stop_after given) the harness's stage-by-stage restatement."""
        w = self.w
        sc = (C.c_float * 3)(*w.scene)
        fl = (C.c_int * 11)(*[int(bool(w.flags.get(n, False))) for n in FLAG_NAMES])
        sizes = (C.c_uint32 * 2)()
        if stop_after is None:
            rc = self.lib.ref_step(sc, C.c_float(w.dt), w.iterations, fl, C.c_float(w.temperature_variation), sizes)
        else:
            rc = self.lib.ref_step_until(sc, C.c_float(w.dt), w.iterations, fl, C.c_float(w.temperature_variation),
                                         stop_after, sizes)
        assert rc == 0
        w.scene = list(sc)
        w.n_sph, w.n_dem = sizes[0], sizes[1]

    def to_host(self):
        w = self.w.copy()
        for s, d in enumerate((w.sph, w.dem, w.bnd, w.buffer)):
            self._copy_set(s, d, False)
        for s, d in enumerate((w.sph_cd, w.dem_cd, w.b_cd)):
            self._copy_cells(s, d, False)
        return w

    def close(self):
        self.lib.ref_destroy()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
