"""ctypes driver for the CPU oracle (TEST INFRASTRUCTURE -- the checker, never the product).

Loads oracle/_build/liboracle{32,64}.so (built by `make -C oracle`) and runs the
restated substep on a HostWorld (snowsimulation_b200.scene) in place.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from snowsimulation_b200.abi import (PARTICLE_FIELDS, CELL_FIELDS, SimParams, flag_bits,
                                     QUIRKS_REFERENCE)

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")


class _Particles(C.Structure):
    _fields_ = [(n, C.c_void_p) for n, _ in PARTICLE_FIELDS]


class _Cells(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in CELL_FIELDS]


class _Scene(C.Structure):
    _fields_ = [("fluid_start_time", C.c_float), ("solid_start_time", C.c_float),
                ("current_time", C.c_float)]


_LIBS = {}


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load(precision=32):
    if precision in _LIBS:
        return _LIBS[precision]
    path = os.path.join(BUILD, "liboracle%d.so" % precision)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    P, PP, CD = C.POINTER(SimParams), C.POINTER(_Particles), _Cells
    u32, pu32 = C.c_uint32, C.POINTER(C.c_uint32)
    lib.or_calculate_hash.argtypes = [P, CD, C.c_void_p, u32]
    lib.or_sort_particles.argtypes = [CD, u32]
    lib.or_reorder_data.argtypes = [CD, C.c_void_p, u32, u32]
    lib.or_compute_boundary_volume.argtypes = [P, CD, C.c_void_p, C.c_void_p, u32]
    lib.or_snow_simulation.argtypes = [P, PP, pu32, PP, pu32, PP, u32, u32, PP, CD, CD, CD,
                                       C.POINTER(_Scene), C.c_float, C.c_int, u32, C.c_float,
                                       C.c_int, C.c_int]
    lib.or_snow_simulation.restype = C.c_int
    lib.or_connect_and_record.argtypes = [P, PP, u32, CD, C.c_int]
    lib.or_energy_momentum.argtypes = [P, PP, u32, PP, u32, C.POINTER(C.c_double)]
    lib.or_set_threads.argtypes = [C.c_int]
    lib.or_set_domain.argtypes = [C.c_float] * 5
    lib.or_real_size.restype = C.c_int
    assert lib.or_real_size() == precision // 8
    _LIBS[precision] = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p).value


class OracleWorld:
    """A HostWorld copy driven through the oracle (precision 32 or 64)."""

    def __init__(self, host_world, precision=32, quirks=QUIRKS_REFERENCE, threads=0):
        self.lib = load(precision)
        if threads:
            self.lib.or_set_threads(int(threads))
        self.precision = precision
        self.quirks = quirks
        w = host_world.copy()
        if precision == 64:
            for d in (w.sph, w.dem, w.bnd, w.buffer, w.sph_cd, w.dem_cd, w.b_cd):
                for k, v in d.items():
                    if v.dtype == np.float32:
                        d[k] = v.astype(np.float64)
        self.w = w
        self.params = w.params
        self.lib.or_set_domain(*[C.c_float(x) for x in w.domain])
        self._structs()

    def _pset(self, d):
        return _Particles(*[_ptr(d[n]) for n, _ in PARTICLE_FIELDS])

    def _cset(self, d):
        return _Cells(*[_ptr(d[n]) for n in CELL_FIELDS])

    def _structs(self):
        w = self.w
        self.p_sph, self.p_dem, self.p_bnd, self.p_buf = (self._pset(w.sph), self._pset(w.dem),
                                                          self._pset(w.bnd), self._pset(w.buffer))
        self.c_sph, self.c_dem, self.c_b = self._cset(w.sph_cd), self._cset(w.dem_cd), self._cset(w.b_cd)

    # -- one-time setup (Simulation::InitializeBoundaryCudaData, Simulation.cpp:558-592)
    def init_boundary(self):
        w, L = self.w, self.lib
        L.or_calculate_hash(C.byref(self.params), self.c_b, _ptr(w.bnd["positions"]), w.n_b)
        L.or_sort_particles(self.c_b, w.n_b)
        L.or_reorder_data(self.c_b, _ptr(w.bnd["positions"]), w.n_b, int(self.params.num_cells))
        L.or_compute_boundary_volume(C.byref(self.params), self.c_b, _ptr(w.bnd["mass"]),
                                     _ptr(w.bnd["volume"]), w.n_b)

    def init_links(self):
        """Form the initial interlinks at rest (one sort of the snow set + connect pass)."""
        w, L = self.w, self.lib
        L.or_calculate_hash(C.byref(self.params), self.c_dem, _ptr(w.dem["predict_positions"]), w.n_dem)
        L.or_sort_particles(self.c_dem, w.n_dem)
        L.or_reorder_data(self.c_dem, _ptr(w.dem["predict_positions"]), w.n_dem, int(self.params.num_cells))
        L.or_connect_and_record(C.byref(self.params), C.byref(self.p_dem), w.n_dem, self.c_dem,
                                int(bool(w.flags.get("dynamic_max_connections"))))

    def setup(self):
        self.init_boundary()
        if self.w.init_links:
            self.init_links()
        return self

    def step(self, stop_after=0, dt=None, iterations=None):
        w = self.w
        self.lib.or_set_domain(*[C.c_float(x) for x in w.domain])
        ns, nd = C.c_uint32(w.n_sph), C.c_uint32(w.n_dem)
        sc = _Scene(*w.scene)
        rc = self.lib.or_snow_simulation(
            C.byref(self.params), C.byref(self.p_sph), C.byref(ns), C.byref(self.p_dem), C.byref(nd),
            C.byref(self.p_bnd), w.n_b, w.full, C.byref(self.p_buf), self.c_sph, self.c_dem, self.c_b,
            C.byref(sc), C.c_float(w.dt if dt is None else dt),
            w.iterations if iterations is None else iterations,
            flag_bits(w.flags), C.c_float(w.temperature_variation), self.quirks, stop_after)
        assert rc == 0
        w.n_sph, w.n_dem = ns.value, nd.value
        w.scene = [sc.fluid_start_time, sc.solid_start_time, sc.current_time]

    def energy_momentum(self):
        out = (C.c_double * 4)()
        self.lib.or_energy_momentum(C.byref(self.params), C.byref(self.p_sph), self.w.n_sph,
                                    C.byref(self.p_dem), self.w.n_dem, out)
        return list(out)
