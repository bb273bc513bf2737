"""Adjoint of the substep (CUDA reverse kernels behind the C-ABI, wrapped in a
torch.autograd.Function) against central finite differences:
  - of the FP64 oracle (the FP64 reference gradient; eps 1e-4 relative for the SimParams
    scalars, which are stored as float32, 1e-5 for the velocity direction): relative
    agreement 1e-3 (observed ~1e-5);
  - of the FP32 GPU forward itself (eps 1e-3 relative): conductivities within 1%; the
    position-driven parameters are below the FP32 loss noise at this eps and are checked
    against the FP64 gradient only.
The scene is small (27 water on 108 snow with interlinks, phase change off) and short
(6 substeps) so that no contact or link event falls inside the FD perturbation."""
import ctypes as C

import numpy as np
import pytest
import torch

from snowsimulation_b200 import scene, _native
from snowsimulation_b200.abi import QUIRKS_FIXED, QUIRKS_REFERENCE, SimParams
from snowsimulation_b200.adjoint import PARAM_NAMES, loss_fn, params_of, restore, rollout, snapshot

pytestmark = pytest.mark.gpu

SUB = 6
W_T = 1e-4


def _setup(flags_off=()):
    from snowsimulation_b200.world import Simulation
    w0 = scene.adjoint_tiny(seed=0)
    for f in flags_off:
        w0.flags[f] = False
    sim = Simulation(w0, quirks=QUIRKS_FIXED).setup()
    start = snapshot(sim)
    theta0 = params_of(sim)
    v0 = sim.sph.t["velocity"][:sim.n_sph].clone()
    v0[:, 1] -= 0.5
    rng = np.random.default_rng(0)
    with torch.no_grad():
        _, xd, _, Td = rollout(sim, v0, theta0, SUB, 10)
    tx = xd + torch.tensor(rng.normal(0, 0.005, size=tuple(xd.shape)), dtype=torch.float32, device=xd.device)
    tT = Td + torch.tensor(rng.normal(0, 1.0, size=tuple(Td.shape)), dtype=torch.float32, device=xd.device)
    restore(sim, start)
    direction = rng.normal(0, 1, size=tuple(v0.shape)).astype(np.float32)
    return w0, sim, start, theta0, v0, tx, tT, direction


def _adjoint(sim, start, theta0, v0, tx, tT, ckpt):
    restore(sim, start)
    vv = v0.clone().requires_grad_(True)
    th = theta0.clone().requires_grad_(True)
    _, xd, _, Td = rollout(sim, vv, th, SUB, ckpt)
    L = loss_fn(xd, Td, tx, tT, W_T)
    L.backward()
    return float(L.detach()), th.grad.numpy().copy(), vv.grad.cpu().numpy().copy()


def _oracle_loss(w0, theta, v, tx64, tT64):
    from oracle.oracle import OracleWorld
    w = w0.copy()
    p = SimParams()
    C.memmove(C.byref(p), C.byref(w0.params), C.sizeof(p))
    for k, n in enumerate(PARAM_NAMES):
        setattr(p, n, float(theta[k]))
    w.params = p
    o = OracleWorld(w, 64, QUIRKS_FIXED).setup()
    o.w.sph["velocity"][:w.n_sph] = v
    for _ in range(SUB):
        o.step()
    x = o.w.dem["positions"][:w.n_dem]
    T = o.w.dem["T"][:w.n_dem]
    return float(((x - tx64) ** 2).sum(1).mean() + W_T * ((T - tT64) ** 2).mean())


@pytest.mark.parametrize("flags_off", [(), ("dem_friction",), ("sph_dem_correction", "dem_viscosity")])
def test_adjoint_matches_fp64_reference_gradient(cuda, flags_off):
    w0, sim, start, theta0, v0, tx, tT, direction = _setup(flags_off)
    L, g_th, g_v = _adjoint(sim, start, theta0, v0, tx, tT, ckpt=4)
    tx64, tT64 = tx.double().cpu().numpy(), tT.double().cpu().numpy()
    v64 = v0.double().cpu().numpy()
    assert abs(_oracle_loss(w0, theta0, v64, tx64, tT64) - L) < 1e-5 * L
    for k in range(4):
        tp, tm = theta0.clone(), theta0.clone()
        tp[k] *= 1 + 1e-4
        tm[k] *= 1 - 1e-4
        step = float(np.float32(tp[k])) - float(np.float32(tm[k]))
        fd = (_oracle_loss(w0, tp, v64, tx64, tT64) - _oracle_loss(w0, tm, v64, tx64, tT64)) / step
        if fd == 0.0:
            assert g_th[k] == 0.0, PARAM_NAMES[k]
        else:
            assert abs(g_th[k] - fd) <= 1e-3 * abs(fd), (PARAM_NAMES[k], g_th[k], fd)
    e = 1e-5
    fd_v = (_oracle_loss(w0, theta0, v64 + e * direction, tx64, tT64)
            - _oracle_loss(w0, theta0, v64 - e * direction, tx64, tT64)) / (2 * e)
    ad_v = float((g_v * direction).sum())
    assert abs(ad_v - fd_v) <= 1e-3 * abs(fd_v), (ad_v, fd_v)


def test_adjoint_conductivities_match_fp32_fd(cuda):
    w0, sim, start, theta0, v0, tx, tT, direction = _setup()
    L, g_th, g_v = _adjoint(sim, start, theta0, v0, tx, tT, ckpt=10)

    def loss(theta):
        restore(sim, start)
        with torch.no_grad():
            _, xd, _, Td = rollout(sim, v0, theta, SUB, 10)
        return float(loss_fn(xd, Td, tx, tT, W_T))

    for k in (2, 3):
        e = 1e-3 * float(theta0[k])
        tp, tm = theta0.clone(), theta0.clone()
        tp[k] += e
        tm[k] -= e
        fd = (loss(tp) - loss(tm)) / (2 * e)
        assert abs(g_th[k] - fd) <= 1e-2 * abs(fd), (PARAM_NAMES[k], g_th[k], fd)


def test_checkpoint_interval_does_not_change_gradients(cuda):
    _, sim, start, theta0, v0, tx, tT, _ = _setup()
    L1, t1, v1 = _adjoint(sim, start, theta0, v0, tx, tT, ckpt=1)
    L2, t2, v2 = _adjoint(sim, start, theta0, v0, tx, tT, ckpt=4)
    L3, t3, v3 = _adjoint(sim, start, theta0, v0, tx, tT, ckpt=100)
    assert L1 == L2 == L3
    # re-recorded segments replay the same forward bit for bit; only the order of the
    # double atomics of the parameter gradients may differ
    assert np.array_equal(v1, v2) and np.array_equal(v1, v3)
    assert np.allclose(t1, t2, rtol=1e-9, atol=0) and np.allclose(t1, t3, rtol=1e-9, atol=0)


def test_rollout_leaves_final_state(cuda):
    _, sim, start, theta0, v0, tx, tT, _ = _setup()
    restore(sim, start)
    vv = v0.clone().requires_grad_(True)
    xs, xd, Ts, Td = rollout(sim, vv, theta0, SUB, 2)
    before = sim.dem.t["positions"].clone()
    loss_fn(xd, Td, tx, tT, W_T).backward()
    assert torch.equal(before, sim.dem.t["positions"])
    assert torch.equal(xd, sim.dem.t["positions"][:sim.n_dem])


def test_recording_rejects_reference_quirks_and_graphs(cuda):
    from snowsimulation_b200.world import Simulation
    lib = _native.load()
    sim = Simulation(scene.adjoint_tiny(seed=1), quirks=QUIRKS_REFERENCE).setup()
    assert lib.snowb_adjoint_begin() == 0
    try:
        with pytest.raises(_native.SnowError, match="FIXED"):
            sim.step()
        sim.quirks = QUIRKS_FIXED
        with pytest.raises(_native.SnowError, match="graph"):
            sim.step(use_graph=True)
    finally:
        n = C.c_uint32(0)
        assert lib.snowb_adjoint_end(C.byref(n)) == 0
    assert n.value == 0


def test_phase_change_while_recording_is_reported(cuda):
    from snowsimulation_b200.world import Simulation
    lib = _native.load()
    w = scene.adjoint_tiny(seed=2)
    w.flags["change_phase"] = True
    w.sph["T"][: w.n_sph] = -5.0      # every water particle freezes in the first substep
    w.sph["new_T"][:] = w.sph["T"]
    sim = Simulation(w, quirks=QUIRKS_FIXED).setup()
    full = sim.full
    bufs = [torch.zeros(full * 3, device=sim.device) for _ in range(6)] + [torch.zeros(full * 25, device=sim.device)]
    io = _native.AdjointIO(*[b.data_ptr() for b in bufs])
    assert lib.snowb_adjoint_begin() == 0
    sim.step()
    n = C.c_uint32(0)
    assert lib.snowb_adjoint_end(C.byref(n)) == 0
    assert n.value == 1
    assert lib.snowb_adjoint_backward(C.byref(io)) == -1
    assert b"phase" in lib.snowb_last_error_string()
