"""Frame export from the GPU: the files hold the device positions of both sets; the
synchronous and asynchronous paths and the host writer produce the same bytes."""
import numpy as np
import pytest

from snowsimulation_b200 import export, scene

pytestmark = pytest.mark.gpu


def test_export_frame_sync_and_async(cuda, tmp_path):
    from snowsimulation_b200.world import Simulation
    sim = Simulation(scene.tiny(seed=3)).setup()
    sim.step(substeps=2)
    H = sim.to_host()
    a = export.export_frame(sim, str(tmp_path / "sync"), 7)
    b = export.export_frame(sim, str(tmp_path / "async"), 7, async_=True)
    export.wait(sim.lib)
    r = float(sim.params.particle_radius)
    for pa, pb, (d, n, rgb, label) in zip(a, b, ((H.sph, H.n_sph, export.WATER_RGB, 0),
                                                 (H.dem, H.n_dem, export.SNOW_RGB, 1))):
        assert open(pa, "rb").read() == open(pb, "rb").read()
        f = export.read_bgeo(pa)
        assert f["n_points"] == n
        assert np.array_equal(f["P"][:, :3], d["positions"][:n])
        ref = str(tmp_path / ("host_%d.bgeo" % label))
        export.write_host(ref, d["positions"][:n], rgb, r, label)
        assert open(ref, "rb").read() == open(pa, "rb").read()
    assert a[0].endswith("frame_7_fluid.bgeo") and a[1].endswith("frame_7_rigid.bgeo")
