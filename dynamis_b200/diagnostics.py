"""Whole-world quantities for judging long runs: energy, momentum and the deepest penetration.

Long runs of a pile are chaotic, so they are not compared state by state; they are held to bounds
on these instead. Everything is computed in float64 on the host from the records the C ABI returns
(BodyStateRecord rows, BodyDescriptorRecord rows, ContactRecords), for the dynamic rows only:
static and kinematic rows have no mass.
"""
from __future__ import annotations

import numpy as np

from . import records as R


def _rotate(q: np.ndarray, v: np.ndarray) -> np.ndarray:
    """v rotated by unit quaternions q (x, y, z, w), row by row."""
    u, w = q[:, :3], q[:, 3:4]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def _dynamic(descs: np.ndarray) -> np.ndarray:
    kinematic = (descs["flags"] & R.BODY_KINEMATIC) != 0
    return (descs["inverse_mass"] > 0) & ~kinematic


def masses(descs: np.ndarray) -> np.ndarray:
    """Per-row mass; 0 for rows that do not simulate."""
    inv = descs["inverse_mass"].astype(np.float64)
    return np.where(_dynamic(descs), 1.0 / np.where(inv > 0, inv, 1.0), 0.0)


def energy(states: np.ndarray, descs: np.ndarray, gravity) -> dict:
    """Kinetic (linear and rotational) and gravitational potential energy of the dynamic rows, J.

    The potential is -m g . x at each body's centre of mass (zero at the origin); the rotational
    part is w^T I w / 2 with I the body's inertia in its own frame and w in that frame."""
    m = masses(descs)
    q = states["orientation"].astype(np.float64)
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    com = states["position"].astype(np.float64) + _rotate(q, descs["com"].astype(np.float64))
    v = states["velocity"].astype(np.float64)
    w = states["angular_velocity"].astype(np.float64)
    conj = q * np.array([-1.0, -1.0, -1.0, 1.0])
    wl = _rotate(conj, w)
    i = descs["inertia"].astype(np.float64)  # xx, xy, xz, yy, yz, zz
    iw = np.stack([i[:, 0] * wl[:, 0] + i[:, 1] * wl[:, 1] + i[:, 2] * wl[:, 2],
                   i[:, 1] * wl[:, 0] + i[:, 3] * wl[:, 1] + i[:, 4] * wl[:, 2],
                   i[:, 2] * wl[:, 0] + i[:, 4] * wl[:, 1] + i[:, 5] * wl[:, 2]], axis=1)
    dyn = m > 0
    linear = 0.5 * np.sum(m * np.sum(v * v, axis=1))
    rotational = 0.5 * np.sum(np.where(dyn, np.sum(wl * iw, axis=1), 0.0))
    g = np.asarray(gravity, np.float64).reshape(3)
    potential = -np.sum(m * (com @ g))
    return {"kinetic_linear": float(linear), "kinetic_rotational": float(rotational),
            "potential": float(potential), "total": float(linear + rotational + potential)}


def momentum(states: np.ndarray, descs: np.ndarray) -> np.ndarray:
    """Total linear momentum of the dynamic rows, kg m/s."""
    m = masses(descs)
    return (m[:, None] * states["velocity"].astype(np.float64)).sum(axis=0)


def deepest_penetration(contacts: np.ndarray) -> float:
    """The largest overlap over the non-sensor contacts' points, m (a point's depth is its overlap:
    positive when the shapes interpenetrate, negative for a speculative point still apart); 0 when
    nothing overlaps."""
    if len(contacts) == 0:
        return 0.0
    live = contacts["sensor"] == 0
    depth = contacts["points"]["depth"].astype(np.float64)
    used = np.arange(4)[None, :] < contacts["point_count"][:, None]
    used &= live[:, None]
    if not used.any():
        return 0.0
    return float(max(0.0, depth[used].max()))


def summary(world, dt: float, stepped: bool = True) -> dict:
    """energy, momentum and deepest_penetration of a World's current state (synchronises).
    Before the world's first step there are no contacts: pass stepped=False."""
    world.wait()
    scene = world.export_scene()
    states = world.read_states()
    descs = scene["descs"]
    gravity = world.step_params(dt)["gravity"][0][:3]
    e = energy(states, descs, gravity)
    p = momentum(states, descs)
    total_mass = float(masses(descs).sum())
    return {"energy": e, "momentum": p.tolist(), "mass": total_mass,
            "mean_velocity": (p / max(total_mass, 1e-30)).tolist(),
            "deepest_penetration": deepest_penetration(world.debug_contacts()) if stepped else 0.0}
