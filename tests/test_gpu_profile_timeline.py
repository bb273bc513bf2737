"""snowb_profile_timeline: the launches of the last profiled substep, one line each with a
start and an end time; an error without profiling."""
import ctypes as C

import pytest

from snowsimulation_b200 import scene

pytestmark = pytest.mark.gpu


def test_profile_timeline(cuda):
    from snowsimulation_b200.world import Simulation
    sim = Simulation(scene.config0()).setup()
    lib = sim.lib
    buf = C.create_string_buffer(1 << 20)
    assert lib.snowb_profile_timeline(buf, len(buf)) != 0      # profiling is off
    sim.step(substeps=2, sync=True, use_graph=True)
    assert lib.snowb_profile_begin() == 0
    sim.step(substeps=2, sync=True, use_graph=True)
    assert lib.snowb_profile_timeline(buf, len(buf)) == 0
    rows = [line.rsplit(None, 2) for line in buf.value.decode().splitlines()]
    summary = C.create_string_buffer(1 << 16)
    assert lib.snowb_profile_end(summary, len(summary)) == 0
    names = [r[0] for r in rows]
    assert "k_density<true>" in names and "k_integrate" in names
    assert all(float(b) >= float(a) for _, a, b in rows)
    # the summary counts two substeps' launches, the timeline one substep's
    counts = {line.rsplit(None, 2)[0]: int(line.rsplit(None, 2)[1]) for line in summary.value.decode().splitlines()}
    assert counts["k_density<true>"] == 2 * names.count("k_density<true>")
