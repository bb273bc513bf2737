"""CUDA path vs the FP32 oracle at the workloads' own horizons (tolerance 0 unless stated).

- config 0 (1,000 water dropped onto 4,096 snow) for its full 120 frames, in both quirk
  modes, compared every 10 frames;
- config 1 (5,888 water + 147,928 snow) for 40 frames, through the dense melt that begins
  near frame 8 (the water sinks into the block and the local neighbour counts reach
  several hundred), compared every 10 frames;
- the temperature-dependent link cap (dynamic_max_connections, adjust_connections,
  cuda_simulation.cu:4768-4816), which is off by default;
- scenes whose water or snow set is empty from the start, and a snow-only scene whose
  melting fills the empty water set;
- the set-up entry points called with zero and one particle;
- the FP64 heat-energy and momentum reductions against the oracle's.
"""
import ctypes as C

import numpy as np
import pytest

from snowsimulation_b200 import scene
from snowsimulation_b200.abi import QUIRKS_REFERENCE, QUIRKS_FIXED
from tests._util import diff_worlds, track_ids

pytestmark = pytest.mark.gpu

SUBSTEPS = 4


def _pair(world, quirks=QUIRKS_REFERENCE):
    from oracle.oracle import OracleWorld
    from snowsimulation_b200.world import Simulation
    o = OracleWorld(world, 32, quirks).setup()
    g = Simulation(world, quirks=quirks).setup()
    return o, g


def _run_frames(o, g, frames, every, what):
    for f in range(1, frames + 1):
        g.step(substeps=SUBSTEPS, use_graph=True)
        for _ in range(SUBSTEPS):
            o.step()
        if f % every == 0 or f == frames:
            d = diff_worlds(o.w, g.to_host())
            assert not d, "%s, frame %d: %s" % (what, f, d[:6])


@pytest.mark.parametrize("quirks", [QUIRKS_REFERENCE, QUIRKS_FIXED])
def test_config0_120_frames_bit_exact(cuda, quirks):
    w = scene.config0()
    o, g = _pair(w, quirks)
    n0 = w.n_sph + w.n_dem
    _run_frames(o, g, 120, 10, "config0")
    assert np.array_equal(track_ids(g.to_host()), np.arange(1, n0 + 1, dtype=np.uint32))


def test_config1_40_frames_through_the_melt_bit_exact(cuda):
    w = scene.config1()
    o, g = _pair(w)
    _run_frames(o, g, 40, 10, "config1")
    # the water has melted into the block by now: the sets have changed size
    assert (g.n_sph, g.n_dem) != (w.n_sph, w.n_dem)


def _dynamic_scene(seed):
    """Snow at temperatures spread over -29..-1 C (caps of 24 down to 0 links), water above
    it; interlinks formed with the dynamic cap at rest."""
    w = scene.tiny(seed=seed, water=(3, 3, 3), snow=(8, 5, 8), drop=0.03, init_links=True)
    rng = np.random.default_rng(seed)
    n = w.n_dem
    w.dem["T"][:n] = rng.uniform(-29.0, -1.0, n).astype(np.float32)
    w.dem["new_T"][:] = w.dem["T"]
    w.flags["dynamic_max_connections"] = True
    return w


@pytest.mark.parametrize("quirks", [QUIRKS_REFERENCE, QUIRKS_FIXED])
def test_dynamic_link_cap_bit_exact(cuda, quirks):
    w = _dynamic_scene(7)
    o, g = _pair(w, quirks)
    _assert = lambda what: (lambda d: (not d) or pytest.fail("%s: %s" % (what, d[:6])))(diff_worlds(o.w, g.to_host()))
    _assert("dynamic links at rest")
    for k in range(8):
        o.step(); g.step()
        _assert("dynamic links, substep %d" % k)
    # the cap is in force: no snow particle holds more links than its temperature allows
    H = g.to_host()
    M, n = H.maxc, H.n_dem
    rec = H.dem["connect_record"][: n * M].reshape(n, M)
    cnt = (rec != 0xFFFFFFFF).sum(1)
    assert cnt.max() > 0
    assert cnt.max() < M


def _one_sided(empty, melt=False):
    water = scene._block((4, 4, 4), 0.02, (0.0, 0.0), 0.3, 0.002, np.random.default_rng(3))
    snow = scene._block((6, 4, 6), 0.02, (0.0, 0.0), 0.01, 0.002, np.random.default_rng(4))
    w = scene.build_world(water[:0] if empty == "water" else water, snow[:0] if empty == "snow" else snow,
                          100.0, -10.0, name="one-sided", init_links=empty != "snow")
    if melt:   # part of the snow above freezing: it melts into the empty water set
        w.dem["T"][:30] = 5.0
        w.dem["new_T"][:] = w.dem["T"]
    return w


@pytest.mark.parametrize("quirks", [QUIRKS_REFERENCE, QUIRKS_FIXED])
@pytest.mark.parametrize("empty,melt", [("water", False), ("snow", False), ("water", True)])
def test_empty_set_from_the_start_bit_exact(cuda, quirks, empty, melt):
    w = _one_sided(empty, melt)
    o, g = _pair(w, quirks)
    for k in range(6):
        o.step(); g.step()
        d = diff_worlds(o.w, g.to_host())
        assert not d, "empty %s, substep %d: %s" % (empty, k, d[:6])
    if melt:
        assert g.n_sph > 0, "the melting snow was meant to fill the water set"


def test_drop_in_calls_with_zero_and_one_particle(cuda):
    """calculate_hash, sort_particles, reorder_data, compute_boundary_volume,
    connect_and_record and integrate_pbd with 0 and 1 particles: status OK, nothing written
    beyond the particles given, and the one-particle results equal the oracle's."""
    import torch
    from snowsimulation_b200 import _native
    from snowsimulation_b200.world import DeviceSet, DeviceCells
    from oracle.oracle import OracleWorld
    lib = _native.load()
    w = scene.tiny(seed=2)
    p = w.params
    _native.check(lib.snowb_set_sim_params(C.byref(p)))
    _native.check(lib.snowb_set_stream(None))
    nc = int(p.num_cells)
    for n in (0, 1):
        ds = DeviceSet(w.dem, cuda)
        dc = DeviceCells(w.dem_cd, cuda)
        s, c = ds.struct(), dc.struct()
        _native.check(lib.snowb_calculate_hash(c, s.predict_positions, n))
        _native.check(lib.snowb_sort_particles(c, n))
        _native.check(lib.snowb_sort_particles_static(c, n))
        _native.check(lib.snowb_reorder_data(c, s.predict_positions, n, nc))
        _native.check(lib.snowb_compute_boundary_volume(c, s.mass, s.volume, n))
        _native.check(lib.snowb_connect_and_record(C.byref(s), n, c, 0))
        _native.check(lib.snowb_integrate_pbd(C.byref(s), C.c_float(w.dt), n, 1))
        torch.cuda.synchronize(cuda)
        G, GC = ds.host(), dc.host()
        # the oracle runs the same calls on the host copy
        o = OracleWorld(w, 32)
        L, W = o.lib, o.w
        from oracle.oracle import _ptr
        L.or_calculate_hash(C.byref(o.params), o.c_dem, _ptr(W.dem["predict_positions"]), n)
        L.or_sort_particles(o.c_dem, n)
        L.or_reorder_data(o.c_dem, _ptr(W.dem["predict_positions"]), n, nc)
        L.or_compute_boundary_volume(C.byref(o.params), o.c_dem, _ptr(W.dem["mass"]), _ptr(W.dem["volume"]), n)
        L.or_connect_and_record(C.byref(o.params), C.byref(o.p_dem), n, o.c_dem, 0)
        for k in ("grid_hash", "grid_index", "cell_start", "cell_end", "sorted_pos"):
            assert np.array_equal(GC[k], W.dem_cd[k]), (n, k)
        for k in ("volume", "connect_record", "iter_end", "connect_length"):
            assert np.array_equal(G[k], W.dem[k]), (n, k)
        # integrate_pbd moves particles [0, n) only
        assert np.array_equal(G["positions"][n:], w.dem["positions"][n:])
        if n == 0:
            assert np.array_equal(G["predict_positions"], w.dem["predict_positions"])


def test_energy_momentum_matches_oracle(cuda):
    """snowb_energy_momentum (FP64 reductions on the GPU) against the oracle's FP64 sums
    over the same state: the terms are the same FP64 products, only the summation order
    differs, so the sums agree to 1e-12 of the summed magnitudes."""
    from oracle.oracle import OracleWorld
    w = scene.config0()
    o, g = _pair(w)
    for _ in range(3 * SUBSTEPS):
        o.step(); g.step()
    assert not diff_worlds(o.w, g.to_host())
    eg = g.energy_momentum()
    eo = o.energy_momentum()
    H = g.to_host()
    mag = [0.0] * 4
    for d, n, c in ((H.sph, H.n_sph, float(w.params.C_water)), (H.dem, H.n_dem, float(w.params.C_snow))):
        m = d["mass"][:n].astype(np.float64)
        mag[0] += float(np.sum(np.abs(m * c * d["T"][:n].astype(np.float64))))
        for k in range(3):
            mag[1 + k] += float(np.sum(np.abs(m * d["velocity"][:n, k].astype(np.float64))))
    for k in range(4):
        assert abs(eg[k] - eo[k]) <= 1e-12 * mag[k] + 1e-300, (k, eg[k], eo[k], mag[k])
    assert eg[0] != 0.0 and mag[2] > 0.0


def test_unchanged_sorts_are_kept_and_stay_bit_exact(cuda):
    """A snow block at rest keeps every particle in its cell, so after the first sort of a
    call the snow set's sort points keep the previous sort (their outputs are kept current
    by the kernels that move the particles); the state stays bit-exact with the oracle,
    which sorts at every sort point."""
    import ctypes as C
    from snowsimulation_b200 import _native
    w = scene.tiny(seed=9, water=(2, 2, 2), snow=(8, 4, 8), drop=0.4, init_links=True)
    o, g = _pair(w)
    for k in range(4):
        o.step(); g.step()
        d = diff_worlds(o.w, g.to_host())
        assert not d, "substep %d: %s" % (k, d[:6])
    g.step(substeps=4)
    for _ in range(4):
        o.step()
    assert not diff_worlds(o.w, g.to_host())
    cnt = (C.c_uint32 * 24)()
    _native.check(g.lib.snowb_device_counters(cnt, 24))
    full_d, kept_d = cnt[21], cnt[23]
    assert kept_d > 0 and full_d + kept_d >= 4 * 7, (full_d, kept_d)
