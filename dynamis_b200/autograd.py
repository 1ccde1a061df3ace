"""A torch.autograd.Function over World::step_backward (the C ABI's dyn_tape_begin / dyn_backward).

`rollout(world, mass, friction, velocity, steps, dt)` steps `world` `steps` times from its current
state with the given per-row masses, per-collider frictions and per-row starting velocities, and
returns the final positions (rows x 3, float32 on the CPU). Its backward reverses the recorded
steps on the device and returns d loss / d mass, d loss / d friction and d loss / d velocity:

* a row's inverse inertia tensor scales with 1 / mass (the shape keeps its mass distribution), so
  d loss / d mass = -(inverse_mass x g_inverse_mass + g_inertia_scale) / mass;
* static rows (mass 0) keep mass 0 and get a zero gradient.

The world keeps the recorded trajectory until the backward (or `release(world)`) ends the tape; after
the backward the world holds the state after the last step again. Torch is needed only here; the
library itself never imports it.
"""
from __future__ import annotations

import numpy as np
import torch

from . import records as R


def _inertia_per_mass(world) -> np.ndarray:
    """The rows' inverse inertia tensors times their masses (constant as the mass changes)."""
    scene = world.export_scene()
    descs = scene["descs"]
    mass = np.where(descs["inverse_mass"] > 0, 1.0 / np.maximum(descs["inverse_mass"], 1e-30), 0.0)
    return descs["inverse_inertia"].astype(np.float64) * mass[:, None], len(scene["colliders"])


class Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mass, friction, velocity, world, steps, dt, checkpoint_interval):
        m = mass.detach().cpu().double().numpy()
        unit, colliders = _inertia_per_mass(world)
        inverse_mass = np.where(m > 0, 1.0 / np.where(m > 0, m, 1.0), 0.0)
        world.set_mass_properties(inverse_mass.astype(np.float32), (unit * inverse_mass[:, None]).astype(np.float32))
        world.set_friction(friction.detach().cpu().numpy().astype(np.float32))
        states = world.read_states()
        states["velocity"] = velocity.detach().cpu().numpy().astype(np.float32)
        world.upload_states(states)
        world.tape_begin(int(checkpoint_interval))
        for _ in range(int(steps)):
            world.step(float(dt))
        final = world.read_states()
        ctx.world = world
        ctx.steps = int(steps)
        ctx.mass = m
        ctx.inverse_mass = inverse_mass
        ctx.colliders = colliders
        return torch.from_numpy(final["position"].astype(np.float32))

    @staticmethod
    def backward(ctx, grad_position):
        world = ctx.world
        n = len(ctx.mass)
        grad = np.zeros(n, R.BODY_GRAD)
        grad["position"] = grad_position.detach().cpu().numpy().astype(np.float32)
        out = world.step_backward(grad, ctx.steps)
        pg = world.param_grads()
        world.tape_end()
        m = ctx.mass
        g_mass = np.where(m > 0, -(ctx.inverse_mass * pg["inverse_mass"] + pg["inertia_scale"]) / np.where(m > 0, m, 1.0), 0.0)
        return (torch.from_numpy(g_mass.astype(np.float32)), torch.from_numpy(pg["friction"].astype(np.float32)),
                torch.from_numpy(out["velocity"].astype(np.float32)), None, None, None, None)


def rollout(world, mass, friction, velocity, steps: int, dt: float, checkpoint_interval: int = 10):
    """Final positions of `steps` steps of `world` (see the module docstring)."""
    return Rollout.apply(mass, friction, velocity, world, steps, dt, checkpoint_interval)


def release(world) -> None:
    """Ends a rollout's tape without a backward (the world returns to the state after its last step)."""
    world.tape_end()
