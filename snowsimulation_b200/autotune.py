"""Launch-shape autotuning of the substep kernels (snowb_autotune in the CUDA library).

tune() runs the library's autotuner on a resident Simulation or BatchSimulation and puts
the state back afterwards; the chosen table can be saved and loaded, so a host tunes once
per GPU model and workload size and reuses the table (kernel, work bucket -> threads per
block, grid cap).  Tuning never changes results, only launch shapes.
"""
import ctypes as C

from . import _native
from .abi import FLAG_NAMES


def _snapshot(sim):
    snap = {"n": (sim.n_sph, sim.n_dem),
            "scene": (sim.scene.fluid_start_time, sim.scene.solid_start_time, sim.scene.current_time),
            "sets": {name: {k: v.clone() for k, v in getattr(sim, name).t.items()}
                     for name in ("sph", "dem", "scd", "dcd")}}
    if hasattr(sim, "sid"):
        snap["sid"] = {k: v.clone() for k, v in sim.sid.items()}
    return snap


def _restore(sim, snap):
    sim.n_sph, sim.n_dem = snap["n"]
    sim.scene.fluid_start_time, sim.scene.solid_start_time, sim.scene.current_time = snap["scene"]
    for name, d in snap["sets"].items():
        for k, v in d.items():
            getattr(sim, name).t[k].copy_(v)
    for k, v in snap.get("sid", {}).items():
        sim.sid[k].copy_(v)


def tune(sim, substeps=3):
    """Tune the kernels for `sim`'s workload; returns the table text."""
    lib = sim.lib
    snap = _snapshot(sim)
    w = sim.w
    ns, nd = C.c_uint32(sim.n_sph), C.c_uint32(sim.n_dem)
    flags = [int(bool(w.flags.get(n, False))) for n in FLAG_NAMES]
    batch = C.byref(sim.batch) if hasattr(sim, "batch") else None
    quirks = getattr(sim, "quirks", 1)
    S = sim._s
    try:
        _native.check(lib.snowb_autotune(
            C.byref(S[0]), C.byref(ns), C.byref(S[1]), C.byref(nd), C.byref(S[2]), sim.n_b, sim.full,
            C.byref(S[3]), sim._c[0], sim._c[1], sim._c[2], C.byref(sim.scene), C.c_float(w.dt), w.iterations,
            *flags, C.c_float(w.temperature_variation), quirks, int(substeps), batch))
    finally:
        _restore(sim, snap)
    return table(lib)


def table(lib=None):
    lib = lib or _native.load()
    buf = C.create_string_buffer(1 << 16)
    _native.check(lib.snowb_autotune_table(buf, len(buf)))
    return buf.value.decode()


def load(text, lib=None):
    lib = lib or _native.load()
    _native.check(lib.snowb_autotune_load(text.encode()))


def reset(lib=None):
    lib = lib or _native.load()
    _native.check(lib.snowb_autotune_reset())


def save_file(path, lib=None):
    with open(path, "w") as f:
        f.write(table(lib))


def load_file(path, lib=None):
    with open(path) as f:
        load(f.read(), lib)
