"""The .bgeo writer (no GPU): header, attribute table, point records and trailer of the
reference's export (GLFWApp::ExportBgeoFile via Partio's classic BGEO writer)."""
import numpy as np

from snowsimulation_b200 import export


def test_bgeo_layout(tmp_path):
    rng = np.random.default_rng(0)
    pos = rng.normal(size=(37, 3)).astype(np.float32)
    path = str(tmp_path / "frame_0_rigid.bgeo")
    export.write_host(path, pos, export.SNOW_RGB, 0.01, export.LABEL_RIGID)
    b = export.read_bgeo(path)
    assert b["magic"] == 0x4267656F and b["version_char"] == b"V" and b["version"] == 5
    assert b["n_points"] == 37 and b["n_prims"] == 0 and b["n_point_attrib"] == 3 and b["n_attrib"] == 0
    assert b["attributes"] == [("Cd", 3, 0), ("pscale", 1, 0), ("label", 1, 1)]
    assert np.array_equal(b["P"][:, :3], pos) and (b["P"][:, 3] == 1.0).all()
    assert np.array_equal(b["Cd"], np.tile(np.float32(export.SNOW_RGB), (37, 1)))
    assert (b["pscale"] == np.float32(0.01)).all()
    # the reference writes the float label's bits into the int attribute
    assert (b["label"] == np.float32(1.0).view(np.uint32)).all()
    assert b["trailer"] == b"\x00\xff"


def test_bgeo_plain_int_label_and_empty(tmp_path):
    path = str(tmp_path / "a.bgeo")
    export.write_host(path, np.zeros((2, 3), np.float32), export.WATER_RGB, 0.01, 1, float_label=False)
    assert (export.read_bgeo(path)["label"] == 1).all()
    path = str(tmp_path / "b.bgeo")
    export.write_host(path, np.zeros((0, 3), np.float32), export.WATER_RGB, 0.01, 0)
    b = export.read_bgeo(path)
    assert b["n_points"] == 0 and b["trailer"] == b"\x00\xff"


def test_host_driver_scene_file_round_trip(tmp_path):
    """The C++ host driver's scene file holds a HostWorld exactly (no GPU involved)."""
    from snowsimulation_b200 import scene
    from snowsimulation_b200.host_io import read_world, write_world
    from tests._util import diff_worlds
    w = scene.tiny(seed=2, init_links=True)
    w.scene = [0.0, 0.5, 0.125]
    p = str(tmp_path / "w.bin")
    write_world(p, w)
    r = read_world(p, w)
    assert not diff_worlds(w, r)
    assert r.scene == w.scene and bytes(r.params) == bytes(w.params)
