"""The FP32 oracle against golden fixtures produced by the reference's own solver
(tests/golden/make_golden.py: cuda_simulation.cu with IEEE arithmetic on a B200, seeded
`tiny` scene, stage boundaries of the first substep).  Tolerance 0: the oracle performs
the same float operations."""
import glob
import os

import numpy as np
import pytest

from oracle.oracle import OracleWorld

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_tiny_stage*.npz")))


def _golden_world():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.skipif(not FILES, reason="no golden fixtures")
@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_oracle_matches_reference_golden(path):
    m = _golden_world()
    stop = int(os.path.basename(path)[len("ref_tiny_stage"):-4])
    o = OracleWorld(m.golden_world(), 32).setup()
    o.step(stop_after=stop)
    got = m.snapshot(o.w)
    ref = dict(np.load(path))
    assert set(got) == set(ref)
    for k in sorted(ref):
        a, b = np.asarray(got[k]), np.asarray(ref[k])
        assert a.shape == b.shape, k
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        assert np.all(same), "%s differs at %d entries" % (k, int((~same).sum()))
