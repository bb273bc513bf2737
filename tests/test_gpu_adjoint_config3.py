"""The adjoint at the adjoint workload's own size: 1,024 water particles falling onto an
8,192-particle snow block with interlinks (phase change off), snow-position loss against a
seeded target (N(0, 0.005 m)) plus a small temperature term, checkpoints every 10
substeps, against central differences of the FP64 oracle.

Horizon and flags, and why.  The loss is only piecewise smooth in the parameters: an
interlink breaks where its length passes 1.05 L (a jump in its force), and friction
switches between its static and kinetic forms (a jump in the correction).  Central
differences that straddle such an event measure the jump, not the derivative, and their
value then changes sign and size with eps (measured on a B200: k_refreezing at 10 frames
gives -2.1e-6, 3.3e-7 and 1.5e-6 for different eps while the adjoint gives 1.4e-7).  With
friction off the workload at frame 10 (40 substeps, the water has reached the block and
heat flows) is smooth in the conductivities, the contact stiffness and the water's initial
velocities over the perturbations used below.  The adjoint follows the FP32 trajectory
and the FP64 differences the FP64 one, which part by up to 1e-4 m by frame 10, so the two
gradients differ where the two trajectories' contact sets do.  Measured on a B200 with this
target: k_water 1.4e-3, k_snow 2.1e-3, the velocity direction 5.7e-4 (eps 1e-6 m/s) and
k_stretch 3.4e-2 (eps 1e-6, the same difference as at eps 1e-4, so no kink in between;
with another seeded target 1.3e-3).  Bounds: 5e-3 for the conductivities, 5e-2 for
k_stretch, 2e-2 for the velocity direction.  k_refreezing is checked on the small scene of
test_gpu_adjoint.py, whose short horizon holds no link-break event.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from snowsimulation_b200 import scene
from snowsimulation_b200.abi import QUIRKS_FIXED, SimParams
from snowsimulation_b200.adjoint import PARAM_NAMES, loss_fn, params_of, restore, rollout, snapshot

pytestmark = pytest.mark.gpu

H = 40          # substeps: frame 10
W_T = 1e-4


def _oracle_loss(w0, theta, v, tx64, tT64):
    import os
    from oracle.oracle import OracleWorld
    w = w0.copy()
    p = SimParams()
    C.memmove(C.byref(p), C.byref(w0.params), C.sizeof(p))
    for k, n in enumerate(PARAM_NAMES):
        setattr(p, n, float(theta[k]))
    w.params = p
    o = OracleWorld(w, 64, QUIRKS_FIXED, threads=os.cpu_count() or 1).setup()
    o.w.sph["velocity"][:w.n_sph] = v
    for _ in range(H):
        o.step()
    assert (o.w.n_sph, o.w.n_dem) == (w0.n_sph, w0.n_dem)
    x = o.w.dem["positions"][:w.n_dem]
    T = o.w.dem["T"][:w.n_dem]
    return float(((x - tx64) ** 2).sum(1).mean() + W_T * ((T - tT64) ** 2).mean())


def test_config3_adjoint_matches_fp64_reference_gradient(cuda):
    from snowsimulation_b200.world import Simulation
    w0 = scene.config3(seed=0)
    w0.flags["dem_friction"] = False
    assert not w0.flags["change_phase"]       # the recording restriction: no phase change
    sim = Simulation(w0, quirks=QUIRKS_FIXED).setup()
    start = snapshot(sim)
    theta0 = params_of(sim)
    v0 = sim.sph.t["velocity"][:sim.n_sph].clone()
    rng = np.random.default_rng(0)
    with torch.no_grad():
        _, xd, _, Td = rollout(sim, v0, theta0, H, 10)
    tx = xd + torch.tensor(rng.normal(0, 0.005, size=tuple(xd.shape)), dtype=torch.float32, device=xd.device)
    tT = Td + torch.tensor(rng.normal(0, 1.0, size=tuple(Td.shape)), dtype=torch.float32, device=xd.device)
    direction = rng.normal(0, 1, size=tuple(v0.shape)).astype(np.float32)
    restore(sim, start)
    vv = v0.clone().requires_grad_(True)
    th = theta0.clone().requires_grad_(True)
    _, xd, _, Td = rollout(sim, vv, th, H, 10)   # raises if a particle changed phase
    L = loss_fn(xd, Td, tx, tT, W_T)
    L.backward()
    g_th, g_v = th.grad.numpy(), vv.grad.cpu().numpy()
    tx64, tT64 = tx.double().cpu().numpy(), tT.double().cpu().numpy()
    v64 = v0.double().cpu().numpy()
    assert abs(_oracle_loss(w0, theta0, v64, tx64, tT64) - float(L)) < 1e-5 * float(L)

    def fd_param(k, eps):
        tp, tm = theta0.clone(), theta0.clone()
        tp[k] *= 1 + eps
        tm[k] *= 1 - eps
        step = float(np.float32(tp[k])) - float(np.float32(tm[k]))
        return (_oracle_loss(w0, tp, v64, tx64, tT64) - _oracle_loss(w0, tm, v64, tx64, tT64)) / step

    rows = []
    for name, eps, tol in (("k_water", 1e-3, 5e-3), ("k_snow", 1e-3, 5e-3), ("k_stretch", 1e-6, 5e-2)):
        k = PARAM_NAMES.index(name)
        fd = fd_param(k, eps)
        rows.append((name, float(g_th[k]), fd, abs(g_th[k] - fd) / abs(fd), tol))
    e = 1e-6   # m/s along a seeded direction (the water starts at rest)
    fd_v = (_oracle_loss(w0, theta0, v64 + e * direction, tx64, tT64)
            - _oracle_loss(w0, theta0, v64 - e * direction, tx64, tT64)) / (2 * e)
    ad_v = float((g_v * direction).sum())
    rows.append(("v_dir", ad_v, fd_v, abs(ad_v - fd_v) / abs(fd_v), 2e-2))
    print("name, adjoint, FP64 central difference, relative error, bound:", rows)
    assert all(r[3] <= r[4] for r in rows), rows
