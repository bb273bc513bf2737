"""CUDA path vs the FP32 oracle: bit-exact state at every stage boundary and after whole
substeps (tolerance 0: both perform the same IEEE FP32 operations in the same order).

Compared state: every array of the water, snow and boundary ParticleDeviceData and all
three CellData (cell tables including their stale entries), except new_index, which both
implementations only use as scratch.
"""
import numpy as np
import pytest

from snowsimulation_b200 import scene
from snowsimulation_b200.abi import QUIRKS_REFERENCE, QUIRKS_FIXED
from tests._util import diff_worlds, track_ids

pytestmark = pytest.mark.gpu

# stage boundaries shared by both implementations (the GPU fuses iteration stages 1-2
# and 3-5, so the comparison inside an iteration happens after 0, 2, 5, 6, 7)
STOPS = [1, 2, 3, 4, 5, 6, 7] + [10 * (1 + it) + k for it in range(3) for k in (0, 2, 5, 6, 7)] + [90, 0]


def _pair(world, quirks):
    from oracle.oracle import OracleWorld
    from snowsimulation_b200.world import Simulation
    o = OracleWorld(world, 32, quirks).setup()
    g = Simulation(world, quirks=quirks).setup()
    return o, g


def phase_scene(seed=3):
    """Water half below freezing, snow partly above: freezing and melting in the first
    substeps, the snow set growing past its launch size (384 < 512)."""
    w = scene.tiny(seed=seed, water=(4, 4, 4), snow=(8, 6, 8), drop=0.01)
    n = w.n_sph
    w.sph["T"][: n // 2] = -1.0
    w.sph["new_T"][:] = w.sph["T"]
    w.dem["T"][: 40] = 2.0
    w.dem["new_T"][:] = w.dem["T"]
    return w


def _assert_same(o, g, what):
    d = diff_worlds(o.w, g.to_host())
    assert not d, "%s: %s" % (what, d[:6])


@pytest.mark.parametrize("quirks", [QUIRKS_REFERENCE, QUIRKS_FIXED])
def test_setup_bit_exact(cuda, quirks):
    o, g = _pair(scene.config0(), quirks)
    _assert_same(o, g, "boundary setup")


@pytest.mark.parametrize("quirks", [QUIRKS_REFERENCE, QUIRKS_FIXED])
@pytest.mark.parametrize("stop", STOPS)
def test_stage_bit_exact(cuda, stop, quirks):
    o, g = _pair(scene.tiny(seed=1), quirks)
    o.step(); g.step()
    o.step(stop_after=stop); g.step(stop_after=stop)
    _assert_same(o, g, "stage %d" % stop)


@pytest.mark.parametrize("quirks", [QUIRKS_REFERENCE, QUIRKS_FIXED])
def test_phase_change_bit_exact(cuda, quirks):
    w = phase_scene()
    o, g = _pair(w, quirks)
    n0 = w.n_sph + w.n_dem
    for k in range(6):
        o.step(); g.step()
        _assert_same(o, g, "phase substep %d" % k)
    # particle conservation (the reference's verification(), cuda_simulation.cu:4303-4384)
    ids = track_ids(g.to_host())
    assert np.array_equal(ids, np.arange(1, n0 + 1, dtype=np.uint32))
    assert o.w.n_dem != w.n_dem, "scene was meant to change phase"


@pytest.mark.parametrize("quirks", [QUIRKS_REFERENCE, QUIRKS_FIXED])
def test_config0_frames_bit_exact(cuda, quirks):
    o, g = _pair(scene.config0(), quirks)
    for k in range(8):   # two frames of 4 substeps
        o.step(); g.step()
    _assert_same(o, g, "config0 after 8 substeps")


def test_config1_substep_bit_exact(cuda):
    """Full config-1 scene, the scale of the reference's published figures (153,816
    particles): initial links and one substep."""
    o, g = _pair(scene.config1(), QUIRKS_REFERENCE)
    _assert_same(o, g, "config1 initial links")
    o.step(); g.step()
    _assert_same(o, g, "config1 substep")


def test_config1_fixed_quirks_substeps_bit_exact(cuda):
    """Config 1 in the fixed-quirk mode: the snow set's XSPH covers all 147,928 snow particles
    (the reference mode limits it to the water set's launch size), which takes the one-thread
    XSPH form above 65,536 particles."""
    o, g = _pair(scene.config1(), QUIRKS_FIXED)
    for k in range(2):
        o.step(); g.step()
        _assert_same(o, g, "config1 fixed, substep %d" % k)


def test_multi_substep_call_matches_single_calls(cuda):
    """substeps=4 in one call (sizes kept on the device) equals four calls."""
    from snowsimulation_b200.world import Simulation
    w = phase_scene(seed=5)
    a = Simulation(w).setup()
    b = Simulation(w).setup()
    for _ in range(4):
        a.step()
    b.step(substeps=4)
    d = diff_worlds(a.to_host(), b.to_host())
    assert not d, d[:6]


def test_graph_replay_matches_direct(cuda):
    """Substeps replayed from a captured CUDA graph equal substeps issued directly."""
    from snowsimulation_b200.world import Simulation
    w = phase_scene(seed=6)
    a = Simulation(w).setup()
    b = Simulation(w).setup()
    a.step(substeps=6)
    b.step(substeps=3, use_graph=True)
    b.step(substeps=3, use_graph=True)
    d = diff_worlds(a.to_host(), b.to_host())
    assert not d, d[:6]


@pytest.mark.parametrize("quirks", [QUIRKS_REFERENCE, QUIRKS_FIXED])
def test_moved_walls_bit_exact(cuda, quirks):
    """snowb_set_domain: walls at x, z = +-0.05 m and the floor at y = 0.01 m squeeze the tiny
    scene, so particles reflect off every wall and the floor; GPU and oracle agree bit for
    bit over four substeps."""
    w = scene.tiny(seed=5)
    w.domain = (-0.05, 0.05, -0.05, 0.05, 0.01)
    o, g = _pair(w, quirks)
    for _ in range(4):
        o.step(); g.step()
    _assert_same(o, g, "moved walls")
    x = g.to_host().dem["positions"][: g.n_dem]
    assert (x[:, 1] >= 0.01).all()


@pytest.mark.parametrize("quirks", [QUIRKS_REFERENCE, QUIRKS_FIXED])
def test_large_water_set_bit_exact(cuda, quirks):
    """More than 65,536 water particles: the water PBF and contact terms take the one-thread
    path instead of the warp-per-particle one (both must match the oracle)."""
    w = scene.scene_drop((42, 42, 42), (10, 4, 10), seed=5, water_jitter=0.002, snow_jitter=0.002,
                         drop_height=0.05, name="large water")
    assert w.n_sph > 65536
    o, g = _pair(w, quirks)
    for k in range(2):
        o.step(); g.step()
        _assert_same(o, g, "substep %d" % k)
