"""Batched scenes on the GPU: every scene of a batched run equals the same scene run
alone (SNOWB_QUIRKS_FIXED), bit for bit, field by field, after several substeps with
phase changes and interlinks; also through CUDA-graph replay."""
import numpy as np
import pytest

from snowsimulation_b200 import scene
from snowsimulation_b200.abi import QUIRKS_FIXED
from snowsimulation_b200.batch import SET_FIELDS, BatchSimulation, scene_state, unpack

pytestmark = pytest.mark.gpu


def _scenes():
    """Four scenes of different sizes; two of them freeze and melt in the first substeps."""
    ws = [scene.tiny(seed=1, init_links=True),
          scene.tiny(seed=2, water=(3, 3, 3), snow=(8, 5, 8), drop=0.02, init_links=True),
          scene.tiny(seed=3, water=(5, 4, 5), snow=(5, 3, 5), drop=0.08, init_links=True),
          scene.tiny(seed=4, water=(2, 2, 2), snow=(6, 6, 6), drop=0.01, init_links=True)]
    w = ws[1]
    w.sph["T"][: w.n_sph // 2] = -1.0
    w.sph["new_T"][:] = w.sph["T"]
    w = ws[3]
    w.dem["T"][:30] = 2.0
    w.dem["new_T"][:] = w.dem["T"]
    return ws


def _alone(w, substeps, use_graph):
    from snowsimulation_b200.world import Simulation
    g = Simulation(w, quirks=QUIRKS_FIXED).setup()
    if use_graph:
        g.step(substeps=substeps, use_graph=True)
    else:
        for _ in range(substeps):
            g.step()
    return scene_state(g.to_host())


def _compare(worlds, bw, sid, alone):
    for s, w in enumerate(worlds):
        got = unpack(bw, sid, s)
        for set_name, a, b in zip(("sph", "dem"), got, alone[s]):
            assert len(a["trackId"]) == len(b["trackId"]), (s, set_name, len(a["trackId"]), len(b["trackId"]))
            for k in SET_FIELDS[set_name]:
                x, y = a[k], b[k]
                same = np.array_equal(x, y, equal_nan=True) if x.dtype.kind == "f" else np.array_equal(x, y)
                assert same, "scene %d %s.%s differs" % (s, set_name, k)


@pytest.mark.parametrize("use_graph", [False, True])
def test_batched_equals_independent(cuda, use_graph):
    worlds = _scenes()
    substeps = 6
    alone = [_alone(w, substeps, use_graph) for w in worlds]
    b = BatchSimulation(worlds).setup()
    if use_graph:
        b.step(substeps=substeps, use_graph=True)
    else:
        for _ in range(substeps):
            b.step()
    bw, sid = b.to_host()
    assert bw.n_sph == sum(len(a[0]["trackId"]) for a in alone)
    assert bw.n_dem == sum(len(a[1]["trackId"]) for a in alone)
    # live particles per scene, counted on the device from the scene ids
    assert b.scene_counts() == ([len(a[0]["trackId"]) for a in alone], [len(a[1]["trackId"]) for a in alone])
    _compare(worlds, bw, sid, alone)


def test_batched_phase_changes_happen(cuda):
    """The batch above is only a meaningful check if particles change set in it."""
    worlds = _scenes()
    b = BatchSimulation(worlds).setup()
    n0 = (b.n_sph, b.n_dem)
    for _ in range(3):
        b.step()
    assert (b.n_sph, b.n_dem) != n0


def test_batched_links_formed(cuda):
    worlds = _scenes()
    b = BatchSimulation(worlds).setup()
    bw, sid = b.to_host()
    links = bw.dem["iter_end"][:bw.n_dem] - np.arange(bw.n_dem, dtype=np.uint32) * np.uint32(bw.maxc)
    assert links.sum() > 0
    for s in range(len(worlds)):
        unpack(bw, sid, s)       # raises on a link that crosses scenes


def test_batched_rejects_reference_quirks(cuda):
    import ctypes as C
    from snowsimulation_b200 import _native
    from snowsimulation_b200.abi import FLAG_NAMES, QUIRKS_REFERENCE
    b = BatchSimulation(_scenes()[:2]).setup()
    w = b.w
    ns, nd = C.c_uint32(b.n_sph), C.c_uint32(b.n_dem)
    opt = _native.StepOptions(QUIRKS_REFERENCE, 1, 0, 0, 1)
    S = b._s
    rc = b.lib.snowb_batch_snow_simulation(
        C.byref(b.batch), C.byref(S[0]), C.byref(ns), C.byref(S[1]), C.byref(nd), C.byref(S[2]), b.n_b, b.full,
        C.byref(S[3]), b._c[0], b._c[1], b._c[2], C.byref(b.scene), C.c_float(w.dt), w.iterations,
        *[1] * len(FLAG_NAMES), C.c_float(0.0), C.byref(opt))
    assert rc == -1
    assert b"FIXED" in b.lib.snowb_last_error_string()


def test_batched_bad_scene_id_reported(cuda):
    """A scene id beyond the batch is masked into range on the device (no out-of-bounds
    access) and reported as a device error."""
    from snowsimulation_b200 import _native
    b = BatchSimulation(_scenes()[:2]).setup()
    b.sid["sph"][0] = 7
    with pytest.raises(_native.SnowError, match="device error"):
        b.step()
