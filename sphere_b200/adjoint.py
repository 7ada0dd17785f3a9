"""Gradients of a DEM run with respect to its contact parameters, for
calibration: a ``torch.autograd.Function`` over the differentiable step of
libsphk (``sph_diff_begin`` / ``sph_diff_backward``).

The run is a scene (a ``Spherebin``, the reference's own scene object) stepped
``steps`` times with contact model 2 in exact FP64 and per-particle friction.
The differentiable inputs are the global normal and tangential stiffness
``k_n`` and ``k_t``, the normal damping ``gamma_n``, a global friction
coefficient ``mu`` and optional per-particle offsets ``dmu`` (particle i has
friction mu + dmu[i]; a contact uses the mean of its two particles').  The
outputs are the final positions and velocities, (np, 3) each, so any loss
written in torch on them (a height profile, a packing fraction) gets its
gradient through ``backward``: the adjoint kernels run every step in
reverse, recomputing each checkpoint segment of ``checkpoint_every`` steps.

There is no CPU path: the forward and the adjoint both run on the GPU.
"""
from __future__ import annotations

import numpy as np
import torch

from .sphk import Simulation
from .state import config_from_spherebin, state_from_spherebin


def _scene_config(sb, k_n, k_t, gamma_n):
    cfg = config_from_spherebin(sb)
    cfg.params = dict(cfg.params)
    cfg.params["k_n"], cfg.params["k_t"], cfg.params["gamma_n"] = float(k_n), float(k_t), float(gamma_n)
    return cfg


def run_forward(sb, steps, k_n, k_t, gamma_n, mu_particle, checkpoint_every=100, device=0,
                graph_steps=None):
    """The differentiable run without autograd: returns the Simulation (left
    in differentiable mode, ready for ``diff_backward``) and the final state."""
    sim = Simulation(_scene_config(sb, k_n, k_t, gamma_n), device=device, graph_steps=graph_steps)
    sim.upload(state_from_spherebin(sb))
    sim.diff_begin(mu=mu_particle, checkpoint_every=checkpoint_every)
    sim.step(steps)
    sim.sync()
    return sim, sim.download()


class DEMRun(torch.autograd.Function):
    """(k_n, k_t, gamma_n, mu, dmu) -> (x_final, v_final)."""

    @staticmethod
    def forward(ctx, k_n, k_t, gamma_n, mu, dmu, sb, steps, checkpoint_every, device):
        mu_p = (float(mu) + dmu.detach().double().cpu().numpy()).astype(np.float64)
        sim, st = run_forward(sb, steps, float(k_n), float(k_t), float(gamma_n), mu_p,
                              checkpoint_every, device)
        ctx.sim = sim
        ctx.dtype = k_n.dtype
        x = torch.from_numpy(st.x[:, :3].copy())
        v = torch.from_numpy(st.vel[:, :3].copy())
        return x, v

    @staticmethod
    def backward(ctx, gx, gv):
        sim = ctx.sim
        try:
            g = sim.diff_backward(None if gx is None else gx.double().cpu().numpy(),
                                  None if gv is None else gv.double().cpu().numpy())
        finally:
            sim.close()
            ctx.sim = None
        t = lambda v: torch.tensor(v, dtype=torch.float64)
        gmu = torch.from_numpy(g["mu"])
        return (t(g["k_n"]), t(g["k_t"]), t(g["gamma_n"]), gmu.sum(), gmu, None, None, None, None)


def simulate(sb, steps, k_n, k_t, gamma_n, mu, dmu=None, checkpoint_every=100, device=0):
    """Final positions and velocities of ``sb`` after ``steps`` differentiable
    steps, as torch tensors that carry gradients to the parameters (0-d
    float64 tensors with requires_grad, or plain numbers)."""
    as_t = lambda v: v if torch.is_tensor(v) else torch.tensor(float(v), dtype=torch.float64)
    if dmu is None:
        dmu = torch.zeros(sb.np, dtype=torch.float64)
    return DEMRun.apply(as_t(k_n), as_t(k_t), as_t(gamma_n), as_t(mu), dmu, sb, int(steps),
                        int(checkpoint_every), int(device))


def height_profile(x, radius, lo, hi, bins=64):
    """Highest sphere top (z + r) in each of ``bins`` equal x-bins over
    [lo, hi); 0 for empty bins.  Differentiable through the maximising
    particle of each bin."""
    r = torch.as_tensor(radius, dtype=x.dtype)
    top = x[:, 2] + r
    b = torch.clamp(((x[:, 0].detach() - lo) / (hi - lo) * bins).long(), 0, bins - 1)
    out = torch.zeros(bins, dtype=x.dtype)
    return out.scatter_reduce(0, b, top, reduce="amax", include_self=True)
