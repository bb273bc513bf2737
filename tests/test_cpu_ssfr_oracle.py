"""Known answers of the screen-space fluid restatement (oracle/ssfr_oracle.py), derived by
hand from the shaders: the sphere depth of a particle straight ahead of the camera, the
thickness at a sprite centre, the bilateral filter on flat and empty depth, and the
composite's pass-through of background and empty pixels."""
import numpy as np

from oracle import ssfr_oracle as so
from snowsimulation_b200 import render

f32 = np.float32


def _mats(cam):
    V = np.asarray(cam.view, f32).reshape(4, 4)          # [col][row]
    P = np.asarray(cam.projection, f32).reshape(4, 4)
    PV = np.zeros((4, 4), f32)
    for c in range(4):
        for r in range(4):
            PV[c][r] = ((P[0][r] * V[c][0] + P[1][r] * V[c][1]) + P[2][r] * V[c][2]) + P[3][r] * V[c][3]
    inv = lambda M: np.linalg.inv(M.T.astype(np.float64)).T.astype(f32).reshape(16)
    return {"PV": PV.reshape(16), "V": V.reshape(16), "P": P.reshape(16), "Pinv": inv(P), "Vinv": inv(V)}


def _cam(w=64, h=48, ps=40.0):
    return render.camera(eye=(0.0, 0.0, 2.0), center=(0.0, 0.0, 0.0), width=w, height=h, point_size=ps)


def test_sphere_depth_of_particle_ahead():
    cam = _cam()
    cd = render.camera_dict(cam)
    m = _mats(cam)
    r = 0.01
    d = so.sphere_depth(m, cd, np.zeros((1, 3), f32), r)
    hit = d < 1
    assert 100 < hit.sum() < 600          # sprite side 40 / 2 = 20 px, a disc of ~314 px
    # nearest point: the sphere's front at eye-space z = -(2 - r)
    P = np.asarray(cam.projection, np.float64).reshape(4, 4)
    ze = -(2.0 - r)
    zc, wc = P[2][2] * ze + P[3][2], P[2][3] * ze
    assert abs(d[hit].min() - zc / wc) < 2e-6
    # depth grows towards the rim of the disc
    assert d[hit].max() > d[hit].min()


def test_thickness_peaks_at_sprite_centre():
    cam = _cam()
    t = so.thickness_fixed(_mats(cam), render.camera_dict(cam), np.zeros((2, 3), f32))
    v = so.thickness_value(t, 0.0)
    assert abs(v.max() - 2 * 0.005) < 5e-5      # two coincident particles, n.z ~ 1 at the centre
    assert (v[t == 0] == 0).all()


def test_bilateral_flat_and_empty():
    d = np.ones((20, 30), f32)
    d[5:15, 10:20] = f32(0.9)
    d[0, 0] = 0
    s = so.smooth(d)
    assert np.array_equal(s[d >= 1], d[d >= 1])
    assert s[0, 0] == 0
    # a flat patch stays flat (equal weights renormalised)
    assert np.abs(s[5:15, 10:20] - f32(0.9)).max() < 1e-6


def test_bilateral_wraps_rows_and_columns():
    d = np.ones((16, 16), f32)
    d[0, :] = f32(0.5)
    d[15, :] = f32(0.7)
    s = so.smooth_pass(d, 2.0, 0.1, 0.0, horizontal=False)   # falloff 0: plain Gaussian along y
    w1 = np.exp(f32(-(f32(0.1) ** 2)))
    # row 0 sees row 15 (wrap) at distance 1 and itself; rows 1, 2, 14 are empty (skipped)
    expect = (f32(0.5) + f32(0.7) * w1) / (f32(1) + w1)
    assert abs(s[0, 3] - expect) < 1e-6


def test_compose_background_and_empty_pixels():
    cam = _cam(16, 12)
    m = _mats(cam)
    D = np.ones((12, 16), f32)
    D[0, 0] = 0
    scene = np.random.default_rng(0).uniform(0, 1, (12, 16, 4)).astype(f32)
    SD = np.ones((12, 16), f32)
    out = so.compose(m, render.camera_dict(cam), D, np.zeros((12, 16), np.uint64), scene, SD)
    assert (out[0, 0] == 0).all()
    assert np.array_equal(out[D == 1], scene[D == 1])
