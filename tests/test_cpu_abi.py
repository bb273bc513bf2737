"""The C-ABI library loads without a GPU and exports every symbol include/*.h declares;
the ctypes mirrors have the C layouts."""
import ctypes as C
import os
import re

from snowsimulation_b200 import _native
from snowsimulation_b200.abi import ParticleDeviceData, CellData, SimParams, SceneParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(snowb_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    from snowsimulation_b200 import build
    build.build()
    lib = _native.load()
    decl = declared_symbols()
    assert len(decl) >= 19
    missing = [n for n in sorted(decl) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_native.EXPORTS) <= decl


def test_struct_layouts():
    assert C.sizeof(ParticleDeviceData) == 24 * 8
    assert C.sizeof(CellData) == 5 * 8
    assert C.sizeof(SimParams) == 46 * 4          # SimParams.h:7-62, all 4-byte members
    assert C.sizeof(SceneParams) == 12


def test_calls_without_params_fail_cleanly():
    lib = _native.load()
    n = C.c_uint32(0)
    t = C.c_uint32(0)
    assert lib.snowb_compute_grid_size(1000, 512, C.byref(n), C.byref(t)) == 0
    assert (n.value, t.value) == (2, 512)
    assert lib.snowb_compute_grid_size(0, 512, C.byref(n), C.byref(t)) == 0
    assert (n.value, t.value) == (0, 0)


def test_autotune_table_round_trip():
    """The autotuner's table parser and printer (no GPU work involved)."""
    import ctypes as C
    lib = _native.load()
    text = "k_density<true> 18 128 16\nk_pbf 18 256 8\nk_link_colour 12 64 64\n"
    assert lib.snowb_autotune_load(text.encode()) == 0
    buf = C.create_string_buffer(4096)
    assert lib.snowb_autotune_table(buf, len(buf)) == 0
    assert buf.value.decode() == text
    for bad in ("k_pbf 18 100 8\n", "k_pbf x 128 8\n", "k_pbf 18 128\n", "k_pbf 99 128 8\n"):
        assert lib.snowb_autotune_load(bad.encode()) != 0
    assert lib.snowb_autotune_table(buf, len(buf)) == 0
    assert buf.value.decode() == text          # a rejected table leaves the old one
    assert lib.snowb_autotune_reset() == 0
    assert lib.snowb_autotune_table(buf, len(buf)) == 0
    assert buf.value.decode() == ""
