"""The reference's host call sequence, in C++ on the reference's own types, runs on a GPU
through the C++ shim: snowsimulation_b200/shim/snow_host.cpp (built with the shim by
oracle/shim_check.sh where the reference's headers are present) allocates the buffers as
ParticleSystem::SetupCUDAMemory does, runs Simulation::InitializeBoundaryCudaData's calls
and then snow_simulation(ParticleSet*, ..., SceneParams&, ...) once per substep as
Simulation::StepCUDA does.  Its final state equals, bit for bit, the state of the same
substeps through the C ABI from Python (ctypes)."""
import os
import subprocess

import pytest

from snowsimulation_b200 import scene
from snowsimulation_b200.host_io import read_world, write_world
from tests._util import diff_worlds

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "shim", "snow_host")
need_driver = pytest.mark.skipif(not os.path.exists(DRIVER), reason="host driver not built (needs the reference's "
                                                                     "headers, oracle/shim_check.sh)")


def _run(world, substeps, tmp_path):
    src, dst = str(tmp_path / "scene.bin"), str(tmp_path / "out.bin")
    write_world(src, world)
    out = subprocess.run([DRIVER, src, dst, str(substeps)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    return read_world(dst, world)


@need_driver
@pytest.mark.parametrize("name,substeps", [("config0", 32), ("phase", 8), ("links", 8)])
def test_host_driver_through_the_shim_matches_the_c_abi(cuda, tmp_path, name, substeps):
    from snowsimulation_b200.world import Simulation
    if name == "config0":       # 8 frames of 1,000 water dropped onto 4,096 snow
        w = scene.config0()
    elif name == "phase":       # freezing and melting in the first substeps
        w = scene.tiny(seed=3, water=(4, 4, 4), snow=(8, 6, 8), drop=0.01)
        w.sph["T"][: w.n_sph // 2] = -1.0
        w.sph["new_T"][:] = w.sph["T"]
        w.dem["T"][:40] = 2.0
        w.dem["new_T"][:] = w.dem["T"]
    else:                       # interlinks formed at rest before the first substep
        w = scene.tiny(seed=4, init_links=True)
    H = _run(w, substeps, tmp_path)
    g = Simulation(w).setup()
    for _ in range(substeps):
        g.step()
    d = diff_worlds(H, g.to_host())
    assert not d, d[:6]
    assert H.scene == g.to_host().scene
