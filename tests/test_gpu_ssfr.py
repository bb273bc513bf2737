"""Screen-space fluid stages (the reference's default view: point_depth, ssfr_thickness,
bilateral and ssfr_fluid shaders as CUDA kernels) against the CPU restatement in
oracle/ssfr_oracle.py: sphere depth and thickness bit for bit; the bilateral smoothing and
the composite, which call exp and pow, within 1e-6 (depth) and 1e-5 (colour) of the
restatement evaluated on the same inputs."""
import ctypes as C

import numpy as np
import pytest
import torch

from snowsimulation_b200 import _native, render, scene
from snowsimulation_b200.export import SNOW_RGB

pytestmark = pytest.mark.gpu

SMOOTH_ATOL = 1e-6
COMPOSE_ATOL = 1e-5


def _sim():
    from snowsimulation_b200.world import Simulation
    sim = Simulation(scene.tiny(seed=4)).setup()
    sim.step(substeps=2)
    return sim


def _cam():
    return render.camera(eye=(0.12, 0.2, 0.4), center=(0.0, 0.05, 0.0), width=96, height=72, point_size=2.0)


def _stages(sim, cam, ss):
    lib = sim.lib
    W, H = cam.width, cam.height
    dev = sim.device
    f = lambda *shape: torch.empty(shape, dtype=torch.float32, device=dev)
    scene_rgba, zb = f(H, W, 4), torch.empty((H, W), dtype=torch.int64, device=dev)
    sdep, fdep, tmp, sm, out = f(H, W), f(H, W), f(H, W), f(H, W), f(H, W, 4)
    thick = torch.empty((H, W), dtype=torch.int64, device=dev)
    a = C.addressof
    pc = render.colour(SNOW_RGB)
    _native.check(lib.snowb_render_clear_colour(a(cam), a(ss.clear_color), scene_rgba.data_ptr(), zb.data_ptr()))
    _native.check(lib.snowb_render_points(C.byref(sim._s[1]), sim.n_dem, a(cam), a(pc), 0, scene_rgba.data_ptr(),
                                          zb.data_ptr()))
    _native.check(lib.snowb_ssfr_clear(a(cam), sdep.data_ptr(), thick.data_ptr()))
    _native.check(lib.snowb_ssfr_clear(a(cam), fdep.data_ptr(), None))
    _native.check(lib.snowb_ssfr_sphere_depth(C.byref(sim._s[1]), sim.n_dem, a(cam), a(ss), sdep.data_ptr()))
    _native.check(lib.snowb_ssfr_sphere_depth(C.byref(sim._s[0]), sim.n_sph, a(cam), a(ss), fdep.data_ptr()))
    _native.check(lib.snowb_ssfr_smooth(a(cam), a(ss), fdep.data_ptr(), tmp.data_ptr(), sm.data_ptr()))
    _native.check(lib.snowb_ssfr_thickness(C.byref(sim._s[0]), sim.n_sph, a(cam), thick.data_ptr()))
    _native.check(lib.snowb_ssfr_compose(a(cam), a(ss), sm.data_ptr(), thick.data_ptr(), scene_rgba.data_ptr(),
                                         sdep.data_ptr(), out.data_ptr()))
    torch.cuda.synchronize()
    cpu = lambda t: t.cpu().numpy()
    return {"scene": cpu(scene_rgba), "sdep": cpu(sdep), "fdep": cpu(fdep), "smooth": cpu(sm),
            "thick": cpu(thick).view(np.uint64), "out": cpu(out)}


@pytest.fixture(scope="module")
def staged(cuda):
    sim = _sim()
    cam = _cam()
    ss = render.ssfr_params(sphere_radius=0.01)
    st = _stages(sim, cam, ss)
    H = sim.to_host()
    mats = render.ssfr_matrices(sim.lib, cam)
    return sim, cam, ss, st, H, mats


def test_sphere_depth_bit_exact(staged):
    from oracle import ssfr_oracle
    sim, cam, ss, st, H, mats = staged
    cd = render.camera_dict(cam)
    ref_w = ssfr_oracle.sphere_depth(mats, cd, H.sph["positions"][:H.n_sph], 0.01)
    ref_s = ssfr_oracle.sphere_depth(mats, cd, H.dem["positions"][:H.n_dem], 0.01)
    assert (st["fdep"] < 1).sum() > 100 and (st["sdep"] < 1).sum() > 500     # both sets in view
    assert np.array_equal(st["fdep"], ref_w)
    assert np.array_equal(st["sdep"], ref_s)


def test_thickness_bit_exact(staged):
    from oracle import ssfr_oracle
    sim, cam, ss, st, H, mats = staged
    ref = ssfr_oracle.thickness_fixed(mats, render.camera_dict(cam), H.sph["positions"][:H.n_sph])
    assert ref.max() > 0
    assert np.array_equal(st["thick"], ref)


def test_smoothing_matches_restatement(staged):
    from oracle import ssfr_oracle
    sim, cam, ss, st, H, mats = staged
    ref = ssfr_oracle.smooth(st["fdep"], 10.0, 0.1, 65.0)
    assert np.array_equal(st["smooth"] >= 1, ref >= 1)
    assert np.abs(st["smooth"] - ref).max() <= SMOOTH_ATOL
    # the filter changes the interior of the water surface
    inner = (st["fdep"] > 0) & (st["fdep"] < 1)
    assert (st["smooth"][inner] != st["fdep"][inner]).any()


def test_compose_matches_restatement(staged):
    from oracle import ssfr_oracle
    sim, cam, ss, st, H, mats = staged
    ref = ssfr_oracle.compose(mats, render.camera_dict(cam), st["smooth"], st["thick"], st["scene"], st["sdep"],
                              light=tuple(ss.light_color), clear=tuple(ss.clear_color))
    water = (st["smooth"] > 0) & (st["smooth"] < st["sdep"]) & (st["smooth"] < 1)
    assert water.sum() > 50
    assert np.allclose(st["out"], ref, rtol=0, atol=COMPOSE_ATOL, equal_nan=True)
    # background pixels show the scene (clear colour where nothing was drawn)
    bg = st["smooth"] >= 1
    assert np.array_equal(st["out"][bg], st["scene"][bg])


def test_render_fluid_equals_stages(staged):
    sim, cam, ss, st, H, mats = staged
    img = render.render_fluid(sim, cam, ss).cpu().numpy()
    assert np.array_equal(img, st["out"])


def test_reference_view_full_size(cuda):
    """The reference's own camera and 1600 x 900 viewport on the 5k-particle scene."""
    from snowsimulation_b200.world import Simulation
    sim = Simulation(scene.config0()).setup()
    sim.step(substeps=4)
    cam = render.reference_camera()
    img = render.render_fluid(sim, cam).cpu().numpy()
    assert img.shape == (900, 1600, 4)
    assert np.isfinite(img).all()
    clear = np.array([0.15, 0.15, 0.15, 0.0], np.float32)
    assert (np.abs(img - clear).max(axis=2) > 0).sum() > 1000     # particles cover part of the view


def test_bad_arguments_are_refused(cuda):
    lib = _native.load()
    cam = _cam()
    ss = render.ssfr_params()
    ss.filter_radius = -1.0
    buf = torch.empty(cam.width * cam.height, dtype=torch.float32, device="cuda")
    rc = lib.snowb_ssfr_smooth(C.addressof(cam), C.addressof(ss), buf.data_ptr(), buf.data_ptr(), buf.data_ptr())
    assert rc != 0
    cam.width = 0
    assert lib.snowb_ssfr_clear(C.addressof(cam), buf.data_ptr(), None) != 0
