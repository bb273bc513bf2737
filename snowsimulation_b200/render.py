"""Headless point-sprite images of the particle sets (the reference's point_sprite shaders,
run as CUDA kernels by libsnowb200; see include/snow_b200.h).

Camera matrices follow glm's conventions (column-major, right-handed, clip depth -1..1), as
the reference's Renderer builds them.  render() draws water and snow of a Simulation into a
device image; save_ppm() writes it as an 8-bit binary PPM (top row first).
"""
import ctypes as C

import numpy as np
import torch

from . import _native
from .export import SNOW_RGB, WATER_RGB

f32 = np.float32


class Camera(C.Structure):
    _fields_ = [("view", C.c_float * 16), ("projection", C.c_float * 16), ("camera_pos", C.c_float * 3),
                ("light_pos", C.c_float * 3), ("point_size", C.c_float), ("width", C.c_uint32),
                ("height", C.c_uint32)]


class PointColour(C.Structure):
    _fields_ = [("rgb", C.c_float * 3), ("use_temperature", C.c_int), ("coolest_rgb", C.c_float * 3),
                ("hottest_rgb", C.c_float * 3), ("coolest_T", C.c_float), ("hottest_T", C.c_float)]


def _norm(v):
    v = np.asarray(v, f32)
    return (v / f32(np.sqrt(f32(np.dot(v, v))))).astype(f32)


def look_at(eye, center, up):
    """glm::lookAt as a column-major 16-vector."""
    eye, center, up = (np.asarray(x, f32) for x in (eye, center, up))
    f = _norm(center - eye)
    s = _norm(np.cross(f, up).astype(f32))
    u = np.cross(s, f).astype(f32)
    M = np.eye(4, dtype=f32)               # M[col][row]
    M[0][0], M[1][0], M[2][0] = s
    M[0][1], M[1][1], M[2][1] = u
    M[0][2], M[1][2], M[2][2] = -f
    M[3][0] = -f32(np.dot(s, eye))
    M[3][1] = -f32(np.dot(u, eye))
    M[3][2] = f32(np.dot(f, eye))
    return M.reshape(16)


def perspective(fovy, aspect, near, far):
    """glm::perspective (right-handed, clip depth -1..1) as a column-major 16-vector."""
    t = f32(np.tan(f32(fovy) / f32(2)))
    M = np.zeros((4, 4), f32)
    M[0][0] = f32(1) / (f32(aspect) * t)
    M[1][1] = f32(1) / t
    M[2][2] = -(f32(far) + f32(near)) / (f32(far) - f32(near))
    M[2][3] = f32(-1)
    M[3][2] = -(f32(2) * f32(far) * f32(near)) / (f32(far) - f32(near))
    return M.reshape(16)


def camera(eye=(0.0, 1.2, 3.0), center=(0.0, 0.3, 0.0), width=640, height=480, fovy=0.8, point_size=400.0,
           light_pos=(0.0, 10.0, 5.0)):
    c = Camera()
    c.view[:] = look_at(eye, center, (0.0, 1.0, 0.0))
    c.projection[:] = perspective(fovy, width / height, 0.05, 50.0)
    c.camera_pos[:] = eye
    c.light_pos[:] = light_pos
    c.point_size = point_size
    c.width, c.height = width, height
    return c


def colour(rgb, temperature=None):
    """Flat colour, or temperature colours ((cool_rgb, hot_rgb, cool_T, hot_T))."""
    pc = PointColour()
    pc.rgb[:] = rgb
    if temperature is not None:
        cool, hot, tc, th = temperature
        pc.use_temperature = 1
        pc.coolest_rgb[:] = cool
        pc.hottest_rgb[:] = hot
        pc.coolest_T, pc.hottest_T = tc, th
    return pc


class SsfrParams(C.Structure):
    _fields_ = [("sphere_radius", C.c_float), ("filter_radius", C.c_float), ("blur_scale", C.c_float),
                ("blur_depth_falloff", C.c_float), ("light_color", C.c_float * 4), ("clear_color", C.c_float * 4)]


def ssfr_params(sphere_radius=0.01, filter_radius=10.0, blur_scale=0.1, blur_depth_falloff=65.0,
                light_color=(1.0, 1.0, 1.0, 0.8), clear_color=(0.15, 0.15, 0.15, 0.0)):
    """The reference Renderer's values (Renderer.cpp:10, :485-690; bilateral_fs.glsl)."""
    p = SsfrParams()
    p.sphere_radius, p.filter_radius, p.blur_scale = sphere_radius, filter_radius, blur_scale
    p.blur_depth_falloff = blur_depth_falloff
    p.light_color[:] = light_color
    p.clear_color[:] = clear_color
    return p


def reference_camera(width=1600, height=900):
    """The reference application's view: CameraDesc of GLFWApp.cpp:176-185 (eye (0, 0, 5)
    looking at the origin, fov 45 handed to glm::perspective as radians, near 0.001, far
    1000), a 1600 x 900 viewport, point size 30 (Renderer.cpp:8-11) and the light at the
    camera (Renderer.cpp:308-309)."""
    c = Camera()
    eye = (0.0, 0.0, 5.0)
    c.view[:] = look_at(eye, (0.0, 0.0, 0.0), (0.0, 1.0, 0.0))
    c.projection[:] = perspective(45.0, f32(width) / f32(height), 0.001, 1000.0)
    c.camera_pos[:] = eye
    c.light_pos[:] = eye
    c.point_size = 30.0
    c.width, c.height = width, height
    return c


def ssfr_matrices(lib, cam):
    """The library's camera matrices: dict of PV, V, P, Pinv, Vinv (16 floats each)."""
    out = (C.c_float * 80)()
    _native.check(lib.snowb_ssfr_matrices(C.addressof(cam), C.addressof(out)))
    a = np.frombuffer(out, np.float32).copy()
    return {k: a[16 * i:16 * i + 16] for i, k in enumerate(("PV", "V", "P", "Pinv", "Vinv"))}


def render_fluid(sim, cam, ssfr=None, snow_colour=None):
    """The reference's default view of `sim` (snow as point sprites, water as a smoothed,
    refracting surface) into a new device image (H x W x 4 float32)."""
    lib = sim.lib
    ss = ssfr if ssfr is not None else ssfr_params(sphere_radius=float(sim.w.params.particle_radius))
    pc = snow_colour if snow_colour is not None else colour(SNOW_RGB)
    nbytes = C.c_uint64(0)
    _native.check(lib.snowb_ssfr_workspace_bytes(C.addressof(cam), C.byref(nbytes)))
    ws = torch.empty(int(nbytes.value) // 4, dtype=torch.float32, device=sim.device)
    img = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device=sim.device)
    _native.check(lib.snowb_render_fluid(C.byref(sim._s[0]), sim.n_sph, C.byref(sim._s[1]), sim.n_dem,
                                         C.addressof(cam), C.addressof(pc), C.addressof(ss), ws.data_ptr(),
                                         img.data_ptr()))
    return img


def render(sim, cam, temperature=None):
    """Water then snow of `sim` into a new device image (H x W x 4 float32)."""
    lib = sim.lib
    img = torch.empty((cam.height, cam.width, 4), dtype=torch.float32, device=sim.device)
    zb = torch.empty((cam.height, cam.width), dtype=torch.int64, device=sim.device)
    zp, ip = zb.data_ptr(), img.data_ptr()
    _native.check(lib.snowb_render_clear(C.addressof(cam), ip, zp))
    for draw, (st, n, rgb) in enumerate(((sim._s[0], sim.n_sph, WATER_RGB), (sim._s[1], sim.n_dem, SNOW_RGB))):
        pc = colour(rgb, temperature)
        _native.check(lib.snowb_render_points(C.byref(st), n, C.addressof(cam), C.addressof(pc), draw, ip, zp))
    return img


def camera_dict(cam):
    """The camera as plain values (for the CPU restatement in the tests)."""
    return {"view": list(cam.view), "projection": list(cam.projection), "camera_pos": list(cam.camera_pos),
            "light_pos": list(cam.light_pos), "point_size": cam.point_size, "width": cam.width,
            "height": cam.height}


def save_ppm(path, img):
    a = img.detach().cpu().numpy() if hasattr(img, "detach") else np.asarray(img)
    rgb = (np.clip(a[::-1, :, :3], 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (rgb.shape[1], rgb.shape[0]))
        f.write(rgb.tobytes())
