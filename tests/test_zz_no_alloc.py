"""The allocation-free sort (snowb_sort_particles_static) against the allocating one.

Some hosts cannot call cudaMalloc once they are running: a render or game loop that
forbids allocation after start-up (cudaMalloc may synchronise the device mid-frame), a
plugin whose host owns every device allocation, a process under a fixed device-memory
budget.  They sort with snowb_sort_particles_static, whose scratch is a static device
array.  This file runs last (pytest collects it last) so a failure here leaves every other
result in place.  Both sorts are integer work, so the comparison is exact (tolerance 0),
and it is made on two calls in a row because the static scratch keeps the previous call's
contents.  The test passes alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from snowsimulation_b200.abi import STATIC_SORT_MAX_PARTICLES, STATIC_SORT_MAX_CELLS

pytestmark = pytest.mark.gpu


def _cells(torch, keys, dev):
    from snowsimulation_b200.abi import CellData
    n = len(keys)
    gh = torch.from_numpy(keys.view(np.int32).copy()).to(dev)
    gi = torch.arange(n, dtype=torch.int32, device=dev)
    return gh, gi, CellData(gh.data_ptr(), gi.data_ptr(), None, None, None)


def test_static_sort_matches_allocating_sort(cuda):
    import torch
    from snowsimulation_b200 import _native
    from snowsimulation_b200.params import make_sim_params
    lib = _native.load()
    p = make_sim_params()
    assert int(p.num_cells) <= STATIC_SORT_MAX_CELLS
    _native.check(lib.snowb_set_sim_params(C.byref(p)))
    _native.check(lib.snowb_set_stream(None))
    rng = np.random.default_rng(11)
    ncells = int(p.num_cells)
    for call, n in enumerate((200_000, 4_097)):
        # clustered keys with many repeats, as cell hashes of a particle block are
        keys = (rng.integers(0, 4000, n) * 61 % ncells).astype(np.uint32)
        a_h, a_i, a_cd = _cells(torch, keys, cuda)
        b_h, b_i, b_cd = _cells(torch, keys, cuda)
        _native.check(lib.snowb_sort_particles(a_cd, n))
        torch.cuda.synchronize(cuda)
        free_before = torch.cuda.mem_get_info(cuda)[0]
        alloc_before = torch.cuda.memory_allocated(cuda)
        reserved_before = torch.cuda.memory_reserved(cuda)
        _native.check(lib.snowb_sort_particles_static(b_cd, n))
        torch.cuda.synchronize(cuda)
        assert torch.cuda.memory_allocated(cuda) == alloc_before
        assert torch.cuda.memory_reserved(cuda) == reserved_before
        if call == 1:   # the module's static array exists after the first call
            assert torch.cuda.mem_get_info(cuda)[0] == free_before
        assert torch.equal(a_h, b_h), "sorted keys differ on call %d" % call
        assert torch.equal(a_i, b_i), "sorted indices differ on call %d" % call
        order = np.argsort(keys, kind="stable").astype(np.int32)
        assert np.array_equal(b_i.cpu().numpy(), order)


def test_static_sort_rejects_oversize(cuda):
    import torch
    from snowsimulation_b200 import _native
    from snowsimulation_b200.params import make_sim_params
    lib = _native.load()
    p = make_sim_params()
    _native.check(lib.snowb_set_sim_params(C.byref(p)))
    n = STATIC_SORT_MAX_PARTICLES + 1
    keys = np.zeros(n, np.uint32)
    _, _, cd = _cells(torch, keys, cuda)
    rc = lib.snowb_sort_particles_static(cd, n)
    assert rc == -1
    assert b"static scratch limit" in lib.snowb_last_error_string()
