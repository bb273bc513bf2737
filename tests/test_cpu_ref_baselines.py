"""The reference's own CPU neighbour search and XPBD distance solver, built from its sources
into oracle/_ref/libsnowcpuref.so for the reported CPU baselines: the harness drives them
as documented (results checked against brute force and a sequential restatement)."""
import numpy as np
import pytest

from oracle import cpu_ref
from snowsimulation_b200 import scene

pytestmark = pytest.mark.skipif(not cpu_ref.available(), reason="libsnowcpuref.so not built")


def test_spatial_search_finds_every_pair_within_h():
    """SpatialSearch keeps j != i with |xi - xj|^2 <= h^2 (NeighborSearch.cpp:236-246)."""
    w = scene.config0()
    p = w.sph["positions"][: w.n_sph].astype(np.float32)
    h = np.float32(0.04)
    pairs, sec = cpu_ref.spatial_search(p, h, calls=2)
    d = p[:, None, :] - p[None, :, :]
    d2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
    assert pairs == int((d2 <= h * h).sum()) - len(p)
    assert sec > 0.0


def _xpbd_restated(pos, a, b, rest, mass, iters):
    """DistanceConstraint::SolveXPBDConstraint (Constraints.cpp) with zero compliance, in
    constraint order, `iters` sweeps (ConstraintSolver.cpp:60-69), FP32."""
    f = np.float32
    x = pos.astype(np.float32).copy()
    w = f(1.0) / f(mass)
    for _ in range(iters):
        for k in range(len(a)):
            i, j = int(a[k]), int(b[k])
            v = x[i] - x[j]
            sq = v * v
            dist = np.sqrt((sq[0] + sq[1]) + sq[2], dtype=np.float32)
            C = dist - rest[k]
            dist = max(dist, f(1e-15))
            dl = (-C - f(0.0) * f(0.0)) / ((w + w) + f(0.0))
            corr = (dl * v) / dist
            x[i] = x[i] + w * corr
            x[j] = x[j] + (-w) * corr
    return x


def test_xpbd_links_match_sequential_restatement():
    rng = np.random.default_rng(3)
    n = 40
    pos = rng.uniform(-0.1, 0.1, (n, 3)).astype(np.float32)
    a = rng.integers(0, n, 120).astype(np.uint32)
    b = ((a + 1 + rng.integers(0, n - 1, 120)) % n).astype(np.uint32)
    d = np.linalg.norm(pos[a] - pos[b], axis=1).astype(np.float32)
    rest = (d * rng.uniform(0.9, 1.1, 120)).astype(np.float32)
    got, sec = cpu_ref.xpbd_links(pos, a, b, rest, mass=0.008, dt=1.0 / 240.0, iters=3, calls=2)
    want = _xpbd_restated(pos, a, b, rest, 0.008, 3)
    assert np.array_equal(got, want)
    # the links are pulled towards their rest lengths
    d_after = np.linalg.norm(got[a] - got[b], axis=1)
    assert np.abs(d_after - rest).mean() < np.abs(d - rest).mean()


def test_link_pairs_from_slots():
    rec = np.full(3 * 4, 0xFFFFFFFF, np.uint32)
    ln = np.zeros(3 * 4, np.float32)
    rec[0], ln[0] = 1, 0.5       # 0-1
    rec[4], ln[4] = 0, 0.5       # 1-0 (same link)
    rec[5], ln[5] = 2, 0.7       # 1-2
    rec[8], ln[8] = 1, 0.7       # 2-1
    a, b, r = cpu_ref.link_pairs(rec, ln, 3, 4)
    assert list(zip(a.tolist(), b.tolist())) == [(0, 1), (1, 2)]
    assert np.allclose(r, [0.5, 0.7])


def test_out_of_range_link_is_refused():
    pos = np.zeros((2, 3), np.float32)
    with pytest.raises(RuntimeError):
        cpu_ref.xpbd_links(pos, [0], [5], [0.1], 0.008, 1.0 / 240.0)
