"""Device-side driver: the host mirror of Simulation::Initialize / Simulation::StepCUDA
(Simulation.cpp:35-172, :174-299) on plain device buffers instead of mapped GL VBOs.

PyTorch only provides device memory and streams; every computation goes through the
C ABI of libsnowb200.so (see include/snow_b200.h).
"""
import ctypes as C

import numpy as np
import torch

from . import _native
from .abi import (PARTICLE_FIELDS, CELL_FIELDS, ParticleDeviceData, CellData, SceneParams,
                  FLAG_NAMES, QUIRKS_REFERENCE)
from .scene import HostWorld

_ND2T = {np.float32: torch.float32, np.float64: torch.float64, np.uint32: torch.int32}


def _to_dev(a, device):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32)).to(device)
    return torch.from_numpy(a).to(device)


def _to_host(t, like):
    a = t.detach().cpu().numpy()
    if like.dtype == np.uint32:
        return a.view(np.uint32).copy()
    return a.copy()


class DeviceSet:
    """Device copy of one ParticleDeviceData (Particle.h:14-52)."""

    def __init__(self, host, device):
        self.like = host
        self.t = {k: _to_dev(v, device) for k, v in host.items()}

    def struct(self):
        return ParticleDeviceData(*[self.t[n].data_ptr() for n, _ in PARTICLE_FIELDS])

    def host(self):
        return {k: _to_host(v, self.like[k]) for k, v in self.t.items()}


class DeviceCells:
    """Device copy of one CellData (NeighborSearch.h:19-26)."""

    def __init__(self, host, device):
        self.like = host
        self.t = {k: _to_dev(v, device) for k, v in host.items()}

    def struct(self):
        return CellData(*[self.t[n].data_ptr() for n in CELL_FIELDS])

    def host(self):
        return {k: _to_host(v, self.like[k]) for k, v in self.t.items()}


class Simulation:
    """A scene resident on the GPU, stepped through libsnowb200."""

    def __init__(self, world: HostWorld, device="cuda", quirks=QUIRKS_REFERENCE):
        self.lib = _native.load()
        dev = torch.device(device)
        if dev.type != "cuda":
            raise _native.SnowError("the solver runs on a CUDA device only")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        torch.cuda.set_device(self.device)
        self.w = world
        self.quirks = quirks
        self.n_sph, self.n_dem, self.n_b, self.full = world.n_sph, world.n_dem, world.n_b, world.full
        self.scene = SceneParams(*world.scene)
        self.sph = DeviceSet(world.sph, self.device)
        self.dem = DeviceSet(world.dem, self.device)
        self.bnd = DeviceSet(world.bnd, self.device)
        self.buf = DeviceSet(world.buffer, self.device)
        self.scd = DeviceCells(world.sph_cd, self.device)
        self.dcd = DeviceCells(world.dem_cd, self.device)
        self.bcd = DeviceCells(world.b_cd, self.device)
        self._s = [self.sph.struct(), self.dem.struct(), self.bnd.struct(), self.buf.struct()]
        self._c = [self.scd.struct(), self.dcd.struct(), self.bcd.struct()]
        self.params = world.params
        _native.check(self.lib.snowb_set_sim_params(C.byref(self.params)))
        _native.check(self.lib.snowb_set_domain(*[C.c_float(x) for x in world.domain]))
        _native.check(self.lib.snowb_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream)))

    # -- Simulation::InitializeBoundaryCudaData (Simulation.cpp:558-592)
    def init_boundary(self):
        L, bc, b = self.lib, self._c[2], self._s[2]
        _native.check(L.snowb_calculate_hash(bc, b.positions, self.n_b))
        _native.check(L.snowb_sort_particles(bc, self.n_b))
        _native.check(L.snowb_reorder_data(bc, b.positions, self.n_b, int(self.params.num_cells)))
        _native.check(L.snowb_compute_boundary_volume(bc, b.mass, b.volume, self.n_b))

    def init_links(self):
        """Initial interlinks at rest: one sort of the snow set and a connect_and_record pass."""
        L, dc, d = self.lib, self._c[1], self._s[1]
        _native.check(L.snowb_calculate_hash(dc, d.predict_positions, self.n_dem))
        _native.check(L.snowb_sort_particles(dc, self.n_dem))
        _native.check(L.snowb_reorder_data(dc, d.predict_positions, self.n_dem, int(self.params.num_cells)))
        _native.check(L.snowb_connect_and_record(C.byref(d), self.n_dem, dc,
                                                 int(bool(self.w.flags.get("dynamic_max_connections")))))

    def setup(self):
        self.init_boundary()
        if self.w.init_links:
            self.init_links()
        torch.cuda.synchronize(self.device)
        return self

    # -- Simulation::StepCUDA (Simulation.cpp:174-299) without the GL map/unmap
    def step(self, substeps=1, stop_after=0, sync=True, dt=None, iterations=None, use_graph=False):
        w = self.w
        ns, nd = C.c_uint32(self.n_sph), C.c_uint32(self.n_dem)
        opt = _native.StepOptions(self.quirks, substeps, stop_after, 1 if use_graph else 0, 1 if sync else 0)
        flags = [int(bool(w.flags.get(n, False))) for n in FLAG_NAMES]
        S = self._s
        _native.check(self.lib.snowb_snow_simulation_ex(
            C.byref(S[0]), C.byref(ns), C.byref(S[1]), C.byref(nd), C.byref(S[2]), self.n_b, self.full,
            C.byref(S[3]), self._c[0], self._c[1], self._c[2], C.byref(self.scene),
            C.c_float(w.dt if dt is None else dt), w.iterations if iterations is None else iterations,
            *flags, C.c_float(w.temperature_variation), C.byref(opt)))
        if sync:
            self.n_sph, self.n_dem = ns.value, nd.value

    def read_sizes(self):
        ns, nd = C.c_uint32(0), C.c_uint32(0)
        _native.check(self.lib.snowb_read_sizes(C.byref(ns), C.byref(nd)))
        self.n_sph, self.n_dem = ns.value, nd.value
        return self.n_sph, self.n_dem

    def energy_momentum(self):
        out = (C.c_double * 4)()
        _native.check(self.lib.snowb_energy_momentum(C.byref(self._s[0]), self.n_sph, C.byref(self._s[1]),
                                                      self.n_dem, out))
        return list(out)

    def to_host(self):
        """Snapshot of the full device state as a HostWorld (checkpoint / comparison)."""
        w = self.w
        torch.cuda.synchronize(self.device)
        return HostWorld(w.params, self.sph.host(), self.dem.host(), self.bnd.host(), self.buf.host(),
                         self.scd.host(), self.dcd.host(), self.bcd.host(), self.n_sph, self.n_dem,
                         self.n_b, self.full, w.maxc,
                         [self.scene.fluid_start_time, self.scene.solid_start_time, self.scene.current_time],
                         w.dt, w.iterations, w.substeps_per_frame, dict(w.flags), w.temperature_variation,
                         w.name, w.init_links, tuple(w.domain))
