"""Batched scenes: many independent HostWorlds stepped as one through libsnowb200.

All scenes share one SimParams (grid, origin, cell size, constants), the step flags, dt,
iterations and scene times.  Their sets are concatenated into one set per kind; a
scene-id array beside each set names each slot's scene, and the library gives every
scene its own block of a wider cell grid (include/snow_b200.h, "batched scenes").

pack()/unpack() are plain numpy and run without a GPU:
  - the live particles [0, n) of each scene are laid end to end, scene after scene;
  - interlink records are index lists into the set, so they are offset by the scene's
    start; iter_end holds i*M + (links of i) and is rebased the same way;
  - unpack() takes the slots of one scene in ascending index order and maps every record
    back to the scene's own indices, so a batched run can be compared field by field with
    the same scene run alone (the library keeps each scene's relative order).
"""
import ctypes as C
import math

import numpy as np
import torch

from . import _native
from .abi import Batch, FLAG_NAMES, QUIRKS_FIXED, SceneParams
from .scene import HostWorld, UMAX, _alloc_cells, _alloc_set
from .world import DeviceCells, DeviceSet, _to_dev, _to_host

# fields compared between a batched scene and the same scene run alone: everything but
# the compaction scratch (scan_index, new_index and predicate hold set-wide positions)
STATE_FIELDS = ("positions", "predict_positions", "new_positions", "velocity", "force", "correction", "mass",
                "massInv", "density", "C", "lambda_", "volume", "T", "new_T", "contrib", "mass_scale",
                "connect_record", "iter_end", "connect_length", "trackId")
# In the water set the interlink records and iter_end are dead data: melting copies a snow
# particle's records along (copy_particle_info, cuda_simulation.cu:3974-4002) and nothing
# reads them until freezing resets them, so they hold snow-set indices of the moment of
# melting and are left out of the water set's state.
SPH_FIELDS = tuple(k for k in STATE_FIELDS if k not in ("connect_record", "iter_end"))
SET_FIELDS = {"sph": SPH_FIELDS, "dem": STATE_FIELDS}


def layout(n_scenes):
    """(scenes_x, scenes_z): powers of two, scenes_x * scenes_z >= n_scenes, as square as possible."""
    total = 1 << max(0, math.ceil(math.log2(max(1, n_scenes))))
    sx = 1 << (int(math.log2(total)) + 1) // 2
    return sx, total // sx


def shard_scenes(sizes, world_size, rank):
    """Indices (ascending) of the scenes that rank `rank` of `world_size` steps.  The scenes
    of a batch are independent, so ranks split them with nothing exchanged inside a step:
    largest first, each scene to the rank holding the fewest particles so far (the lowest
    rank on a tie).  The split depends on the scene sizes alone, so every rank computes the
    same one without communicating; every scene lands on exactly one rank, and a rank may
    get none when there are fewer scenes than ranks."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("rank %r outside a world of %r" % (rank, world_size))
    load = [0] * world_size
    mine = []
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world_size), key=lambda q: (load[q], q))
        load[r] += int(sizes[i])
        if r == rank:
            mine.append(i)
    return sorted(mine)


def _check_compatible(worlds):
    w0 = worlds[0]
    for w in worlds[1:]:
        if bytes(w.params) != bytes(w0.params):
            raise ValueError("batched scenes must share SimParams")
        same = (w.maxc == w0.maxc and w.dt == w0.dt and w.iterations == w0.iterations
                and w.flags == w0.flags and w.temperature_variation == w0.temperature_variation
                and list(w.scene) == list(w0.scene) and w.init_links == w0.init_links
                and tuple(w.domain) == tuple(w0.domain))
        if not same:
            raise ValueError("batched scenes must share maxc, dt, iterations, flags, scene times and init_links")


def _pack_set(sets, counts, full, maxc, fill_like):
    """Concatenate the live slots [0, n_s) of each scene's set into one set of `full` slots."""
    out = _alloc_set(full, maxc)
    # the padding looks like build_world's padding
    out["positions"][:] = np.inf
    out["predict_positions"][:] = np.inf
    out["new_positions"][:] = np.inf
    out["mass"][:] = fill_like["mass"][0]
    out["massInv"][:] = fill_like["massInv"][0]
    out["contrib"][:] = 1.0
    out["mass_scale"][:] = 1.0
    out["iter_end"][:] = np.arange(full, dtype=np.uint32) * np.uint32(maxc)
    off = 0
    for s, n in zip(sets, counts):
        for k, v in s.items():
            if k in ("new_end", "connect_record", "connect_length", "iter_end"):
                continue
            out[k][off:off + n] = v[:n]
        rec = s["connect_record"][:n * maxc].copy()
        rec[rec != UMAX] += np.uint32(off)
        out["connect_record"][off * maxc:(off + n) * maxc] = rec
        out["connect_length"][off * maxc:(off + n) * maxc] = s["connect_length"][:n * maxc]
        links = s["iter_end"][:n] - np.arange(n, dtype=np.uint32) * np.uint32(maxc)
        out["iter_end"][off:off + n] = (np.arange(off, off + n, dtype=np.uint32) * np.uint32(maxc) + links)
        off += n
    out["new_end"][0] = off
    return out


def pack(worlds):
    """One HostWorld holding every scene, plus the scene-id arrays (sph, dem, boundary)."""
    _check_compatible(worlds)
    w0 = worlds[0]
    maxc = w0.maxc
    full = int(sum(w.full for w in worlds))
    ns = [w.n_sph for w in worlds]
    nd = [w.n_dem for w in worlds]
    nb = [w.n_b for w in worlds]
    sph = _pack_set([w.sph for w in worlds], ns, full, maxc, w0.sph)
    dem = _pack_set([w.dem for w in worlds], nd, full, maxc, w0.dem)
    n_b = int(sum(nb))
    bnd = _pack_set([w.bnd for w in worlds], nb, n_b, maxc, w0.bnd)
    buffer = _alloc_set(full, maxc)

    def ids(counts, size):
        a = np.zeros(size, np.uint32)
        a[:sum(counts)] = np.repeat(np.arange(len(counts), dtype=np.uint32), counts)
        return a

    sid = dict(sph=ids(ns, full), dem=ids(nd, full), bnd=ids(nb, n_b))
    sx, sz = layout(len(worlds))
    nc = int(w0.params.num_cells) * sx * sz
    w = HostWorld(w0.params, sph, dem, bnd, buffer, _alloc_cells(full, nc), _alloc_cells(full, nc),
                  _alloc_cells(n_b, nc), int(sum(ns)), int(sum(nd)), n_b, full, maxc, list(w0.scene),
                  w0.dt, w0.iterations, w0.substeps_per_frame, dict(w0.flags), w0.temperature_variation,
                  "batch of %d scenes" % len(worlds), w0.init_links, tuple(w0.domain))
    return w, sid


def _unpack_set(d, sid, n, scene, maxc, fields):
    idx = np.nonzero(sid[:n] == scene)[0].astype(np.uint32)
    m = len(idx)
    local = np.full(max(n, 1), UMAX, np.uint32)
    local[idx] = np.arange(m, dtype=np.uint32)
    out = {}
    for k in fields:
        v = d[k]
        if k == "connect_record":
            rec = v[:n * maxc].reshape(-1, maxc)[idx]
            live = rec != UMAX
            if live.any():
                tgt = rec[live]
                if (tgt >= n).any() or (sid[tgt] != scene).any():
                    raise AssertionError("scene %d holds a link into another scene or the tail" % scene)
                rec = rec.copy()
                rec[live] = local[tgt]
            out[k] = rec.reshape(-1)
        elif k == "connect_length":
            out[k] = v[:n * maxc].reshape(-1, maxc)[idx].reshape(-1)
        elif k == "iter_end":
            links = v[idx] - idx * np.uint32(maxc)
            out[k] = np.arange(m, dtype=np.uint32) * np.uint32(maxc) + links
        else:
            out[k] = v[idx]
    return out


def unpack(world, sid, scene):
    """The live water and snow particles of one scene, in the scene's own indexing:
    (sph_fields, dem_fields) with SPH_FIELDS and STATE_FIELDS."""
    M = world.maxc
    return (_unpack_set(world.sph, sid["sph"], world.n_sph, scene, M, SPH_FIELDS),
            _unpack_set(world.dem, sid["dem"], world.n_dem, scene, M, STATE_FIELDS))


def scene_state(world):
    """The same view of a scene run alone: live slots of STATE_FIELDS."""
    M = world.maxc
    out = []
    for d, n, fields in ((world.sph, world.n_sph, SPH_FIELDS), (world.dem, world.n_dem, STATE_FIELDS)):
        out.append({k: (d[k][:n * M] if k in ("connect_record", "connect_length") else d[k][:n]) for k in fields})
    return tuple(out)


class BatchSimulation:
    """Many scenes resident on the GPU and stepped together (SNOWB_QUIRKS_FIXED)."""

    def __init__(self, worlds, device="cuda"):
        self.lib = _native.load()
        dev = torch.device(device)
        if dev.type != "cuda":
            raise _native.SnowError("the solver runs on a CUDA device only")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        torch.cuda.set_device(dev)
        self.n_scenes = len(worlds)
        self.w, sid = pack(worlds)
        w = self.w
        self.n_sph, self.n_dem, self.n_b, self.full = w.n_sph, w.n_dem, w.n_b, w.full
        self.scene = SceneParams(*w.scene)
        self.sph, self.dem = DeviceSet(w.sph, dev), DeviceSet(w.dem, dev)
        self.bnd, self.buf = DeviceSet(w.bnd, dev), DeviceSet(w.buffer, dev)
        self.scd, self.dcd, self.bcd = DeviceCells(w.sph_cd, dev), DeviceCells(w.dem_cd, dev), DeviceCells(w.b_cd, dev)
        self.sid = {k: _to_dev(v, dev) for k, v in sid.items()}
        self.sid["buf"] = torch.zeros_like(self.sid["sph"])
        self._sid_like = sid
        sx, sz = layout(self.n_scenes)
        self.batch = Batch(sx, sz, self.sid["sph"].data_ptr(), self.sid["dem"].data_ptr(),
                           self.sid["bnd"].data_ptr(), self.sid["buf"].data_ptr())
        self._s = [self.sph.struct(), self.dem.struct(), self.bnd.struct(), self.buf.struct()]
        self._c = [self.scd.struct(), self.dcd.struct(), self.bcd.struct()]
        _native.check(self.lib.snowb_set_sim_params(C.byref(w.params)))
        _native.check(self.lib.snowb_set_domain(*[C.c_float(x) for x in w.domain]))
        _native.check(self.lib.snowb_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        nc = C.c_uint32(0)
        _native.check(self.lib.snowb_batch_num_cells(C.byref(self.batch), C.byref(nc)))
        assert nc.value == len(w.sph_cd["cell_start"])

    def setup(self):
        L, B = self.lib, C.byref(self.batch)
        bc, b = self._c[2], self._s[2]
        _native.check(L.snowb_batch_calculate_hash(B, bc, b.positions, self.batch.scene_boundary, self.n_b))
        _native.check(L.snowb_batch_sort_particles(B, bc, self.n_b))
        _native.check(L.snowb_batch_reorder_data(B, bc, b.positions, self.n_b))
        _native.check(L.snowb_batch_compute_boundary_volume(B, bc, b.mass, b.volume, self.n_b))
        if self.w.init_links:
            dc, d = self._c[1], self._s[1]
            _native.check(L.snowb_batch_calculate_hash(B, dc, d.predict_positions, self.batch.scene_dem, self.n_dem))
            _native.check(L.snowb_batch_sort_particles(B, dc, self.n_dem))
            _native.check(L.snowb_batch_reorder_data(B, dc, d.predict_positions, self.n_dem))
            _native.check(L.snowb_batch_connect_and_record(B, C.byref(d), self.n_dem, dc,
                                                           int(bool(self.w.flags.get("dynamic_max_connections")))))
        torch.cuda.synchronize(self.device)
        return self

    def step(self, substeps=1, sync=True, use_graph=False, stop_after=0):
        w = self.w
        ns, nd = C.c_uint32(self.n_sph), C.c_uint32(self.n_dem)
        opt = _native.StepOptions(QUIRKS_FIXED, substeps, stop_after, 1 if use_graph else 0, 1 if sync else 0)
        flags = [int(bool(w.flags.get(n, False))) for n in FLAG_NAMES]
        S = self._s
        _native.check(self.lib.snowb_batch_snow_simulation(
            C.byref(self.batch), C.byref(S[0]), C.byref(ns), C.byref(S[1]), C.byref(nd), C.byref(S[2]), self.n_b,
            self.full, C.byref(S[3]), self._c[0], self._c[1], self._c[2], C.byref(self.scene), C.c_float(w.dt),
            w.iterations, *flags, C.c_float(w.temperature_variation), C.byref(opt)))
        if sync:
            self.n_sph, self.n_dem = ns.value, nd.value

    def read_sizes(self):
        ns, nd = C.c_uint32(0), C.c_uint32(0)
        _native.check(self.lib.snowb_read_sizes(C.byref(ns), C.byref(nd)))
        self.n_sph, self.n_dem = ns.value, nd.value
        return self.n_sph, self.n_dem

    def scene_counts(self):
        """(water, snow) live particles per scene, counted on the device from the scene ids."""
        torch.cuda.synchronize(self.device)
        out = []
        for k, n in (("sph", self.n_sph), ("dem", self.n_dem)):
            ids = self.sid[k][:n].long()
            out.append([int(x) for x in torch.bincount(ids, minlength=self.n_scenes).cpu()])
        return tuple(out)

    def to_host(self):
        """(HostWorld of the concatenated sets, scene-id arrays)."""
        torch.cuda.synchronize(self.device)
        w = self.w
        hw = HostWorld(w.params, self.sph.host(), self.dem.host(), self.bnd.host(), self.buf.host(),
                       self.scd.host(), self.dcd.host(), self.bcd.host(), self.n_sph, self.n_dem, self.n_b,
                       self.full, w.maxc, [self.scene.fluid_start_time, self.scene.solid_start_time,
                                           self.scene.current_time],
                       w.dt, w.iterations, w.substeps_per_frame, dict(w.flags), w.temperature_variation,
                       w.name, w.init_links, tuple(w.domain))
        sid = {k: _to_host(self.sid[k], self._sid_like[k]) for k in ("sph", "dem", "bnd")}
        return hw, sid
