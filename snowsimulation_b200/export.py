"""Frame export as Houdini .bgeo files, as GLFWApp::ExportBgeoFile does (GLFWApp.cpp:287-405):
one file per set and frame, point attributes position, Cd, pscale and label.

export_frame() writes `frame_<k>_fluid.bgeo` and `frame_<k>_rigid.bgeo` from a resident
Simulation through the library (positions copied to pinned memory, then written; with
async=True a host thread writes the files while the GPU goes on, and wait() joins them).
read_bgeo() parses such a file back (used by the tests and handy for checks).
"""
import ctypes as C
import os
import struct

import numpy as np

from . import _native

WATER_RGB = (0.7, 0.7, 1.0)      # Simulation.cpp:629/694, opt 0
SNOW_RGB = (0.85, 0.85, 0.85)    # opt 1
LABEL_FLUID, LABEL_RIGID = 0, 1


def _rgb(c):
    return (C.c_float * 3)(*c)


def export_frame(sim, directory, frame, async_=False, float_label=True):
    """Both sets of `sim` at its current state; returns the two paths."""
    lib = sim.lib
    os.makedirs(directory, exist_ok=True)
    r = float(sim.params.particle_radius)
    fn = lib.snowb_export_bgeo_async if async_ else lib.snowb_export_bgeo
    paths = []
    for name, st, n, rgb, label in (("fluid", sim._s[0], sim.n_sph, WATER_RGB, LABEL_FLUID),
                                    ("rigid", sim._s[1], sim.n_dem, SNOW_RGB, LABEL_RIGID)):
        path = os.path.join(directory, "frame_%d_%s.bgeo" % (frame, name))
        _native.check(fn(C.byref(st), n, path.encode(), _rgb(rgb), C.c_float(r), label, int(bool(float_label))))
        paths.append(path)
    return paths


def wait(lib=None):
    lib = lib or _native.load()
    _native.check(lib.snowb_export_wait())


def write_host(path, positions, rgb, pscale, label, float_label=True, lib=None):
    """The library's writer on host positions (n x 3 float32); needs no GPU."""
    lib = lib or _native.load()
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    _native.check(lib.snowb_write_bgeo_host(pos.ctypes.data_as(C.c_void_p), len(pos), path.encode(), _rgb(rgb),
                                            C.c_float(pscale), int(label), int(bool(float_label))))


def read_bgeo(path):
    """Parse a classic (V5) .bgeo with point attributes only: returns a dict with the header
    counts, 'P' (n x 4 float32, homogeneous) and one array per attribute."""
    with open(path, "rb") as f:
        data = f.read()
    o = 0

    def take(fmt):
        nonlocal o
        v = struct.unpack_from(">" + fmt, data, o)
        o += struct.calcsize(">" + fmt)
        return v

    magic, = take("i")
    ver_char, = take("c")
    version, = take("i")
    n_points, n_prims, n_pgroups, n_prgroups, n_pattr, n_vattr, n_prattr, n_attr = take("8i")
    out = dict(magic=magic, version_char=ver_char, version=version, n_points=n_points, n_prims=n_prims,
               n_point_groups=n_pgroups, n_prim_groups=n_prgroups, n_point_attrib=n_pattr,
               n_vertex_attrib=n_vattr, n_prim_attrib=n_prattr, n_attrib=n_attr)
    attrs = []
    for _ in range(n_pattr):
        ln, = take("h")
        name = data[o:o + ln].decode()
        o += ln
        count, htype = take("Hi")
        take("%di" % count)
        attrs.append((name, count, htype))
    width = 4 + sum(c for _, c, _ in attrs)
    words = np.frombuffer(data, dtype=">u4", count=n_points * width, offset=o).reshape(n_points, width)
    o += n_points * width * 4
    out["P"] = words[:, :4].view(">f4").astype(np.float32)
    col = 4
    for name, count, htype in attrs:
        w = words[:, col:col + count]
        out[name] = w.view(">f4").astype(np.float32) if htype in (0, 5) else w.astype(np.uint32)
        col += count
    out["attributes"] = attrs
    out["trailer"] = data[o:]
    return out
