"""CPU checks of the oracle (known-answer cases derived by hand from the reference's
formulas), the scene builder and FP32-vs-FP64 agreement."""
import math

import numpy as np
import pytest

from snowsimulation_b200 import scene
from snowsimulation_b200.params import make_sim_params
from oracle.oracle import OracleWorld


def _world(water, snow, T_water=100.0, T_snow=-10.0, **kw):
    return scene.build_world(np.asarray(water, np.float32).reshape(-1, 3),
                             np.asarray(snow, np.float32).reshape(-1, 3), T_water, T_snow, **kw)


def test_boundary_box_count():
    # InitializeBoundaryParticles with r = 0.01: 102*102 floor + 2*101*102 + 2*104*101
    b = scene.boundary_box(0.01)
    assert len(b) == 102 * 102 + 2 * 101 * 102 + 2 * 104 * 101 == 52016
    assert np.isclose(b[:, 1].min(), -0.02, atol=1e-6)


def test_config_sizes():
    w0 = scene.config0()
    assert (w0.n_sph, w0.n_dem, w0.full) == (1000, 4096, 5096)
    w1 = scene.config1()
    assert (w1.n_sph, w1.n_dem) == (5888, 147928)
    assert np.all(np.abs(w1.dem["positions"][: w1.n_dem, [0, 2]]) < 1.0)


def test_kernel_constants():
    p = make_sim_params()
    h = 0.04
    assert math.isclose(p.poly6, 315.0 / (64 * math.pi * h ** 9), rel_tol=1e-6)
    assert math.isclose(p.spiky_G, -45.0 / (math.pi * h ** 6), rel_tol=1e-6)
    assert math.isclose(p.scorr_divisor, 315.0 / (64 * math.pi * h ** 9) * (h * h - 0.09 * h * h) ** 3, rel_tol=1e-5)


def test_density_two_particles_kat():
    """Two snow particles 0.02 m apart, far from the walls' boundary layer:
    rho = m W(0) + m W(0.02) (compute_snow_dem_sph_density_d, :2320-2423)."""
    p = make_sim_params()
    far = [5.0, 5.0, 5.0]   # water particle far away
    w = _world([far], [[0.3, 0.5, 0.3], [0.32, 0.5, 0.3]], params=p)
    o = OracleWorld(w, 64).setup()
    o.step(stop_after=2)
    h, m = float(np.float32(0.04)), float(w.dem["mass"][0])
    d = float(np.float32(0.32)) - float(np.float32(0.3))
    W = lambda d: float(p.poly6) * (h * h - d * d) ** 3
    expect = m * W(0.0) + m * W(d)
    assert math.isclose(o.w.dem["density"][0], expect, rel_tol=1e-9)
    assert math.isclose(o.w.dem["C"][0], max(expect / 1000.0 - 1.0, 0.0), rel_tol=1e-9, abs_tol=1e-12)


def test_interlink_pair_correction_kat():
    """One link stretched by 10 %: correction = k_ref * -w0/(w0+w1) * (d-L) * n (:4661-4739)."""
    p = make_sim_params()
    w = _world([[5.0, 5.0, 5.0]], [[0.3, 0.5, 0.3], [0.33, 0.5, 0.3]], params=p)
    L = 0.03 / 1.04
    M = w.maxc
    w.dem["connect_record"][0] = 1; w.dem["connect_length"][0] = L
    w.dem["connect_record"][M] = 0; w.dem["connect_length"][M] = L
    w.dem["iter_end"][0] += 1; w.dem["iter_end"][1] += 1
    w.flags["dem_friction"] = False
    w.flags["use_interlink"] = True
    o = OracleWorld(w, 64).setup()
    o.step(stop_after=7)                 # after integrate (gravity moved both equally)
    pp = o.w.dem["predict_positions"][:2].astype(np.float64)
    o.step(stop_after=15)                # first iteration through the interlink stage
    d = np.linalg.norm(pp[0] - pp[1])
    n = (pp[0] - pp[1]) / (d + 0.01 * 0.01)
    expect = 0.75 * -0.5 * (d - L) * n
    # the snow pair also gets density/contact terms: both are zero at 0.03 m > 2r and the
    # PBF term vanishes when C = 0 (two particles are below rest density)
    got = o.w.dem["correction"][0]
    assert np.allclose(got, expect, rtol=1e-6, atol=1e-12)


def test_heat_exchange_two_particles_kat():
    """Water at 100 C next to snow at -10 C (transfer_heat_sph/dem, :3812-3937, own-cell quirk)."""
    p = make_sim_params()
    # both in the same grid cell so the reference's own-cell-only sum sees the pair
    w = _world([[0.405, 0.505, 0.405]], [[0.415, 0.505, 0.405]], params=p)
    o = OracleWorld(w, 64).setup()
    o.step(stop_after=3)
    h, d = float(np.float32(0.04)), float(np.float32(0.415)) - float(np.float32(0.405))
    m, rho_w, rho_s = float(w.sph["mass"][0]), float(o.w.sph["density"][0]), float(o.w.dem["density"][0])
    lap = float(p.viscosity_laplacian) * (h - d)
    kws = 4 * 600.0 * 2500.0 / 3100.0
    dt = float(np.float32(w.dt))
    dTw = 27 * (m / rho_s) * kws * (-10.0 - 100.0) * lap / (4182.0 * rho_w)
    dTs = 27 * (m / rho_w) * kws * (100.0 + 10.0) * lap / (2090.0 * rho_s)
    assert math.isclose(o.w.sph["T"][0], 100.0 + dTw * dt, rel_tol=1e-9)
    assert math.isclose(o.w.dem["T"][0], -10.0 + dTs * dt, rel_tol=1e-9)


def test_neighbor_count_lattice_site():
    """An interior site of the 0.02 m lattice has 26 neighbours closer than h = 0.04 m
    (the 3x3x3 block; the 6 at exactly 2 spacings are not < h), so link formation caps at 25."""
    w = scene.scene_drop((2, 2, 2), (7, 7, 7), drop_height=0.5)
    o = OracleWorld(w, 32).setup()
    o.init_links()
    M = w.maxc
    counts = (o.w.dem["connect_record"][: w.n_dem * M].reshape(-1, M) != 0xFFFFFFFF).sum(1)
    pos = w.dem["positions"][: w.n_dem]
    centre = np.argmin(np.linalg.norm(pos - pos.mean(0), axis=1))
    assert counts[centre] == 25
    assert counts.max() <= 25


def test_links_symmetric_and_unique():
    w = scene.config0()
    o = OracleWorld(w, 32).setup()
    o.init_links()
    M = w.maxc
    rec = o.w.dem["connect_record"][: w.n_dem * M].reshape(-1, M)
    pairs = set()
    for i in range(w.n_dem):
        js = rec[i][rec[i] != 0xFFFFFFFF]
        assert len(js) == len(set(js.tolist()))
        for j in js:
            assert i in rec[j]
            pairs.add((min(i, j), max(i, j)))
    assert len(pairs) > 0


def test_fp32_vs_fp64_small():
    w = scene.tiny(seed=2)
    a = OracleWorld(w, 32).setup()
    b = OracleWorld(w, 64).setup()
    for _ in range(4):
        a.step(); b.step()
    n = a.w.n_dem
    assert (a.w.n_sph, a.w.n_dem) == (b.w.n_sph, b.w.n_dem)
    err = np.abs(a.w.dem["positions"][:n] - b.w.dem["positions"][:n]).max()
    assert err < 5e-5, err
    terr = np.abs(a.w.sph["T"][: a.w.n_sph] - b.w.sph["T"][: a.w.n_sph]).max()
    assert terr < 1e-3, terr


def test_phase_change_conserves_particles():
    """verification() (cuda_simulation.cu:4303-4384): track ids 1..N stay unique."""
    w = scene.tiny(seed=4, drop=0.01)
    w.sph["T"][: w.n_sph // 2] = -1.0
    w.sph["new_T"][:] = w.sph["T"]
    w.dem["T"][:30] = 3.0
    w.dem["new_T"][:] = w.dem["T"]
    o = OracleWorld(w, 32).setup()
    for _ in range(3):
        o.step()
    ids = np.sort(np.concatenate([o.w.sph["trackId"][: o.w.n_sph], o.w.dem["trackId"][: o.w.n_dem]]))
    assert np.array_equal(ids, np.arange(1, w.full + 1, dtype=np.uint32))
    assert (o.w.n_sph, o.w.n_dem) != (w.n_sph, w.n_dem)


def test_domain_default_is_reference_and_floor_moves():
    """The default domain of a world is the reference's box (walls +-1 m, floor 0); a raised
    floor holds the particles above it (the integrate step clamps to floor + r)."""
    from snowsimulation_b200 import scene
    from snowsimulation_b200.abi import QUIRKS_FIXED
    from oracle.oracle import OracleWorld
    assert tuple(scene.tiny().domain) == (-1.0, 1.0, -1.0, 1.0, 0.0)
    w = scene.tiny(seed=2)
    w.domain = (-1.0, 1.0, -1.0, 1.0, 0.03)
    o = OracleWorld(w, 32, QUIRKS_FIXED).setup()
    for _ in range(3):
        o.step()
    y = o.w.dem["positions"][: o.w.n_dem, 1]
    assert y.min() >= 0.03 - 1e-6
    o2 = OracleWorld(scene.tiny(seed=2), 32, QUIRKS_FIXED).setup()
    for _ in range(3):
        o2.step()
    assert o2.w.dem["positions"][: o2.w.n_dem, 1].min() < 0.03


@pytest.mark.parametrize("empty", ["water", "snow"])
def test_empty_set_substeps(empty):
    """A scene whose water or snow set is empty from the start steps through whole
    substeps (its sorts see zero particles); the other set stays finite and keeps its size."""
    snow = [[0.3 + 0.02 * i, 0.5, 0.3] for i in range(8)]
    water = [[0.02 * i, 0.3, 0.0] for i in range(8)]
    w = _world([] if empty == "water" else water, [] if empty == "snow" else snow)
    o = OracleWorld(w, 64).setup()
    for _ in range(3):
        o.step()
    ns, nd = o.w.n_sph, o.w.n_dem
    assert (ns, nd) == ((0, 8) if empty == "water" else (8, 0))
    live = o.w.dem["positions"][:nd] if empty == "water" else o.w.sph["positions"][:ns]
    assert np.all(np.isfinite(live))
