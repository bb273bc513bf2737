"""Host side of batched scenes: scene layout, the pack/unpack of particle sets
(interlink records and iter_end rebased per scene) and the split of a batch's scenes
between ranks."""
import numpy as np
import pytest

from snowsimulation_b200 import scene
from snowsimulation_b200.batch import layout, pack, unpack, scene_state, shard_scenes, SET_FIELDS
from snowsimulation_b200.scene import UMAX


@pytest.mark.parametrize("n,expect", [(1, (1, 1)), (2, (2, 1)), (3, (2, 2)), (4, (2, 2)), (5, (4, 2)),
                                      (8, (4, 2)), (64, (8, 8)), (100, (16, 8))])
def test_layout_powers_of_two(n, expect):
    sx, sz = layout(n)
    assert (sx, sz) == expect
    assert sx * sz >= n


def _linked_world(seed, **kw):
    w = scene.tiny(seed=seed, **kw)
    M, n = w.maxc, w.n_dem
    rng = np.random.default_rng(seed)
    # a few symmetric links so the rebasing of records and iter_end is exercised
    for _ in range(3 * n):
        i, j = rng.integers(0, n, 2)
        if i == j:
            continue
        ci = w.dem["iter_end"][i] - i * M
        cj = w.dem["iter_end"][j] - j * M
        if ci >= M or cj >= M:
            continue
        w.dem["connect_record"][i * M + ci] = j
        w.dem["connect_record"][j * M + cj] = i
        w.dem["connect_length"][i * M + ci] = 0.01
        w.dem["connect_length"][j * M + cj] = 0.01
        w.dem["iter_end"][i] += 1
        w.dem["iter_end"][j] += 1
    return w


def test_pack_unpack_round_trip():
    worlds = [_linked_world(1), _linked_world(2, water=(3, 3, 3), snow=(5, 5, 5)), _linked_world(3, snow=(4, 2, 4))]
    bw, sid = pack(worlds)
    assert bw.n_sph == sum(w.n_sph for w in worlds)
    assert bw.n_dem == sum(w.n_dem for w in worlds)
    assert bw.full == sum(w.full for w in worlds)
    assert len(bw.sph_cd["cell_start"]) == int(worlds[0].params.num_cells) * 4
    for s, w in enumerate(worlds):
        got = unpack(bw, sid, s)
        want = scene_state(w)
        for name, a, b in zip(("sph", "dem"), got, want):
            assert set(a) == set(SET_FIELDS[name]) == set(b)
            for k in SET_FIELDS[name]:
                assert np.array_equal(a[k], b[k]), (s, k)


def test_pack_offsets_records():
    worlds = [_linked_world(1), _linked_world(2)]
    bw, sid = pack(worlds)
    M, off = bw.maxc, worlds[0].n_dem
    rec = bw.dem["connect_record"][off * M:(off + worlds[1].n_dem) * M]
    live = rec[rec != UMAX]
    assert live.size and live.min() >= off and live.max() < off + worlds[1].n_dem
    links = bw.dem["iter_end"][:bw.n_dem] - np.arange(bw.n_dem, dtype=np.uint32) * np.uint32(M)
    assert np.array_equal(links, np.concatenate([w.dem["iter_end"][:w.n_dem] - np.arange(w.n_dem, dtype=np.uint32) * np.uint32(M)
                                                 for w in worlds]))


def test_unpack_rejects_cross_scene_link():
    worlds = [_linked_world(1), _linked_world(2)]
    bw, sid = pack(worlds)
    M = bw.maxc
    bw.dem["connect_record"][0] = np.uint32(worlds[0].n_dem + 1)   # scene 0 -> scene 1
    with pytest.raises(AssertionError):
        unpack(bw, sid, 0)


def test_pack_rejects_mixed_params():
    from snowsimulation_b200.params import make_sim_params
    a = scene.tiny(seed=1)
    b = scene.tiny(seed=2, params=make_sim_params(grid_size=(32, 64, 64)))
    with pytest.raises(ValueError):
        pack([a, b])


def test_config2_shape():
    ws = scene.config2(seed=0)
    n = np.array([w.n_sph + w.n_dem for w in ws])
    assert len(ws) == 64
    assert n.min() >= 1500 and n.max() <= 45000
    frac = np.array([w.n_sph / (w.n_sph + w.n_dem) for w in ws])
    assert frac.min() > 0.005 and frac.max() < 0.4
    assert all(w.init_links for w in ws)
    assert len({bytes(w.params) for w in ws}) == 1


@pytest.mark.parametrize("ws", [1, 2, 3, 4, 8])
def test_shard_scenes_covers_each_scene_once(ws):
    sizes = [w.n_sph + w.n_dem for w in scene.config2(seed=0)]
    parts = [shard_scenes(sizes, ws, r) for r in range(ws)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(sizes)))
    for p in parts:
        assert p == sorted(p)
    # largest first to the lightest rank: no rank is heavier than the lightest by more
    # than the largest scene
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)
    # the same split on every call (each rank computes it alone)
    assert parts == [shard_scenes(sizes, ws, r) for r in range(ws)]


def test_shard_scenes_more_ranks_than_scenes():
    sizes = [30, 10, 20]
    parts = [shard_scenes(sizes, 5, r) for r in range(5)]
    assert parts == [[0], [2], [1], [], []]


def test_shard_scenes_equal_sizes_in_index_order():
    assert [shard_scenes([5] * 6, 3, r) for r in range(3)] == [[0, 3], [1, 4], [2, 5]]


@pytest.mark.parametrize("ws,rank", [(0, 0), (2, 2), (2, -1)])
def test_shard_scenes_rejects_bad_rank(ws, rank):
    with pytest.raises(ValueError):
        shard_scenes([1, 2], ws, rank)
