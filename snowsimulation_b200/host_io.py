"""The scene file of the C++ host driver (snowsimulation_b200/shim/snow_host.cpp).

Layout (little endian, no padding): the magic "SNOWHST1"; u32 n_sph, n_dem, n_b, full,
maxc, num_cells, iterations, init_links, flags (bit i = abi.FLAG_NAMES[i]); f32 dt,
temperature_variation; SimParams (SimParams.h:7-62); SceneParams (SceneParams.h:4-9); then
every array of the water, snow and boundary sets and the phase-change buffer, member by
member in ParticleDeviceData order (Particle.h:14-52), and of the water, snow and boundary
CellData (NeighborSearch.h:19-26), raw.
"""
import ctypes as C
import struct

import numpy as np

from .abi import PARTICLE_FIELDS, CELL_FIELDS, SimParams, flag_bits
from .scene import HostWorld

MAGIC = b"SNOWHST1"
_HEAD = struct.Struct("<8s9I2f")


def _sets(w):
    return (w.sph, w.dem, w.bnd, w.buffer)


def _cells(w):
    return (w.sph_cd, w.dem_cd, w.b_cd)


def write_world(path, w: HostWorld):
    with open(path, "wb") as f:
        f.write(_HEAD.pack(MAGIC, w.n_sph, w.n_dem, w.n_b, w.full, w.maxc, int(w.params.num_cells), w.iterations,
                           1 if w.init_links else 0, flag_bits(w.flags), w.dt, w.temperature_variation))
        f.write(bytes(w.params))
        f.write(struct.pack("<3f", *w.scene))
        for s in _sets(w):
            for name, _ in PARTICLE_FIELDS:
                f.write(np.ascontiguousarray(s[name]).tobytes())
        for c in _cells(w):
            for name in CELL_FIELDS:
                f.write(np.ascontiguousarray(c[name]).tobytes())


def read_world(path, like: HostWorld) -> HostWorld:
    """The state in a scene file, shaped like `like` (same sizes of arrays)."""
    w = like.copy()
    with open(path, "rb") as f:
        magic, ns, nd, nb, full, maxc, ncells, iters, links, flags, dt, dtv = _HEAD.unpack(f.read(_HEAD.size))
        assert magic == MAGIC and (nb, full, maxc) == (w.n_b, w.full, w.maxc)
        w.params = SimParams.from_buffer_copy(f.read(C.sizeof(SimParams)))
        w.scene = list(struct.unpack("<3f", f.read(12)))
        w.n_sph, w.n_dem = ns, nd
        for s in _sets(w):
            for name, _ in PARTICLE_FIELDS:
                a = s[name]
                s[name] = np.frombuffer(f.read(a.nbytes), a.dtype).reshape(a.shape).copy()
        for c in _cells(w):
            for name in CELL_FIELDS:
                a = c[name]
                c[name] = np.frombuffer(f.read(a.nbytes), a.dtype).reshape(a.shape).copy()
        assert f.read(1) == b""
    return w
