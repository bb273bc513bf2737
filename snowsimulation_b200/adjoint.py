"""Differentiable rollouts of the substep: a thin torch.autograd.Function over the adjoint
entry points of libsnowb200 (include/snow_b200.h, "adjoint of the substep").

Forward: `substeps` substeps of a Simulation (fixed quirks) from the current state, with
the water particles' initial velocities and four SimParams scalars (k_refreezing,
k_stretch, k_water, k_snow) as inputs; outputs are the final positions and temperatures
of both sets.  Memory is bounded by checkpointing: the forward keeps a device snapshot of
the state every `checkpoint_every` substeps and nothing else; the backward walks the
segments last to first, restores the segment's snapshot, re-runs it with the tape on and
runs the library's reverse pass over it.

All derivative arithmetic is in the CUDA library; torch only holds device buffers.
"""
import ctypes as C

import torch

from . import _native
from .abi import QUIRKS_FIXED

PARAM_NAMES = ("k_refreezing", "k_stretch", "k_water", "k_snow")
# what the substep rewrites (the rest of a set is constant while no phase changes)
_STATE_FIELDS = ("positions", "predict_positions", "new_positions", "velocity", "correction", "density", "C",
                 "lambda_", "T", "new_T", "contrib", "connect_record", "connect_length", "iter_end", "predicate",
                 "scan_index", "new_end", "trackId")


def snapshot(sim):
    """Device copy of the mutable solver state of a Simulation (checkpoint)."""
    snap = {"n": (sim.n_sph, sim.n_dem),
            "scene": (sim.scene.fluid_start_time, sim.scene.solid_start_time, sim.scene.current_time)}
    for name in ("sph", "dem"):
        ds = getattr(sim, name)
        snap[name] = {k: ds.t[k].clone() for k in _STATE_FIELDS}
    return snap


def restore(sim, snap):
    sim.n_sph, sim.n_dem = snap["n"]
    sim.scene.fluid_start_time, sim.scene.solid_start_time, sim.scene.current_time = snap["scene"]
    for name in ("sph", "dem"):
        ds = getattr(sim, name)
        for k, v in snap[name].items():
            ds.t[k].copy_(v)


def set_params(sim, theta):
    """Write the differentiable SimParams scalars (theta, 4 values) into the library."""
    p = sim.params
    for k, name in enumerate(PARAM_NAMES):
        setattr(p, name, float(theta[k]))
    _native.check(sim.lib.snowb_set_sim_params(C.byref(p)))


def params_of(sim):
    return torch.tensor([float(getattr(sim.params, n)) for n in PARAM_NAMES], dtype=torch.float64)


def _run(sim, substeps):
    for _ in range(substeps):
        sim.step()


class Rollout(torch.autograd.Function):
    """(v_sph0, theta) -> (x_sph, x_dem, T_sph, T_dem) after `substeps` substeps."""

    @staticmethod
    def forward(ctx, v_sph0, theta, sim, substeps, checkpoint_every):
        if sim.quirks != QUIRKS_FIXED:
            raise _native.SnowError("differentiable rollouts need the fixed quirk mode")
        ns, nd = sim.n_sph, sim.n_dem
        set_params(sim, theta)
        sim.sph.t["velocity"][:ns].copy_(v_sph0.to(sim.sph.t["velocity"]))
        C_ = max(1, int(checkpoint_every))
        checkpoints = []
        done = 0
        while done < substeps:
            checkpoints.append(snapshot(sim))
            k = min(C_, substeps - done)
            _run(sim, k)
            done += k
        if (sim.n_sph, sim.n_dem) != (ns, nd):
            raise _native.SnowError("particles changed phase during a differentiable rollout")
        ctx.sim, ctx.substeps, ctx.C, ctx.checkpoints = sim, substeps, C_, checkpoints
        ctx.theta = theta.detach().clone()
        ctx.final = snapshot(sim)
        out = (sim.sph.t["positions"][:ns].clone(), sim.dem.t["positions"][:nd].clone(),
               sim.sph.t["T"][:ns].clone(), sim.dem.t["T"][:nd].clone())
        return out

    @staticmethod
    def backward(ctx, gx_sph, gx_dem, gT_sph, gT_dem):
        sim = ctx.sim
        ns, nd, full = sim.n_sph, sim.n_dem, sim.full
        dev = sim.device
        bufs = {}
        for name, n, g, width in (("gx_sph", ns, gx_sph, 3), ("gx_dem", nd, gx_dem, 3), ("gT_sph", ns, gT_sph, 1),
                                  ("gT_dem", nd, gT_dem, 1), ("gv_sph", ns, None, 3), ("gv_dem", nd, None, 3)):
            t = torch.zeros((full, width) if width == 3 else (full,), dtype=torch.float32, device=dev)
            if g is not None:
                t[:n] = g.to(torch.float32).reshape(t[:n].shape)
            bufs[name] = t
        # adjoint of the interlink rest lengths, carried across segments
        bufs["gL_dem"] = torch.zeros(full * sim.w.maxc, dtype=torch.float32, device=dev)
        io = _native.AdjointIO(*[bufs[k].data_ptr() for k in ("gx_sph", "gv_sph", "gT_sph", "gx_dem", "gv_dem",
                                                              "gT_dem", "gL_dem")])
        set_params(sim, ctx.theta)
        lib = sim.lib
        for seg in range(len(ctx.checkpoints) - 1, -1, -1):
            restore(sim, ctx.checkpoints[seg])
            k = min(ctx.C, ctx.substeps - seg * ctx.C)
            _native.check(lib.snowb_adjoint_begin())
            try:
                _run(sim, k)
            finally:
                rec = C.c_uint32(0)
                _native.check(lib.snowb_adjoint_end(C.byref(rec)))
            _native.check(lib.snowb_adjoint_backward(C.byref(io)))
        restore(sim, ctx.final)
        g_theta = torch.tensor(list(io.grad_params), dtype=torch.float64)
        g_v = bufs["gv_sph"][:ns].clone()
        return g_v, g_theta, None, None, None


def rollout(sim, v_sph0, theta, substeps, checkpoint_every=10):
    """Differentiable rollout; see Rollout."""
    return Rollout.apply(v_sph0, theta, sim, substeps, checkpoint_every)


def loss_fn(x_dem, T_dem, target_x, target_T=None, w_T=0.0):
    """Mean squared distance of the snow positions to a target (plus an optional weighted
    mean squared temperature error, which brings the conductivities into the loss)."""
    L = ((x_dem.double() - target_x.double()) ** 2).sum(dim=1).mean()
    if target_T is not None and w_T:
        L = L + w_T * ((T_dem.double() - target_T.double()) ** 2).mean()
    return L
