"""Point-sprite rendering (the reference's point_sprite shaders as CUDA kernels) against
the CPU restatement in oracle/render_oracle.py, bit for bit: flat colours for water and
snow in one image (depth test across draws), and the temperature colours."""
import numpy as np
import pytest

from snowsimulation_b200 import render, scene
from snowsimulation_b200.export import SNOW_RGB, WATER_RGB

pytestmark = pytest.mark.gpu


def _sim():
    from snowsimulation_b200.world import Simulation
    sim = Simulation(scene.tiny(seed=4)).setup()
    sim.step(substeps=2)
    return sim


def test_render_matches_oracle(cuda):
    from oracle import render_oracle
    sim = _sim()
    cam = render.camera(eye=(0.15, 0.25, 0.45), center=(0.0, 0.05, 0.0), width=96, height=64, point_size=2.5)
    img = render.render(sim, cam).cpu().numpy()
    H = sim.to_host()
    ref = render_oracle.render(render.camera_dict(cam),
                               [(H.sph["positions"][:H.n_sph], None, {"rgb": WATER_RGB}),
                                (H.dem["positions"][:H.n_dem], None, {"rgb": SNOW_RGB})])
    assert (img[..., 3] > 0).sum() > 500          # the scene is in view
    assert np.array_equal(img, ref)


def test_render_temperature_colours(cuda):
    from oracle import render_oracle
    sim = _sim()
    cam = render.camera(eye=(-0.3, 0.2, 0.35), center=(0.0, 0.05, 0.0), width=80, height=80, point_size=2.5)
    t = ((0.0, 0.0, 1.0), (1.0, 0.0, 0.0), -20.0, 100.0)
    img = render.render(sim, cam, temperature=t).cpu().numpy()
    H = sim.to_host()
    ref = render_oracle.render(render.camera_dict(cam),
                               [(H.sph["positions"][:H.n_sph], H.sph["T"][:H.n_sph], {"temperature": t}),
                                (H.dem["positions"][:H.n_dem], H.dem["T"][:H.n_dem], {"temperature": t})])
    assert (img[..., 3] > 0).sum() > 500
    assert np.array_equal(img, ref)
