"""The FP64 reference gradient of the differentiable step, pinned on the CPU.

oracle/adjoint64.cpp restates the solve, integration and position passes in FP64 over the frozen
contact sets of a trajectory recorded with the FP32 oracle. Here its forward-mode derivatives are
checked against its own central differences (h = 1e-4 relative, the step the device gradient check
uses), and its forward against the FP32 oracle's trajectory, on two small tower worlds (sleeping off)
struck by a sphere. These pin the reference the device adjoint (dyn_step_backward) is checked against.
"""
import numpy as np
import pytest

from dynamis_b200 import World, records as R, scenes
from oracle import adjoint as A
from oracle.oracle import OracleWorld

DT = 1.0 / 120.0


def tower_batch(levels=2, footprint=2, worlds=2, seed=3, distance=2.2, heading=None, gap=0.0):
    rng = np.random.default_rng(seed)
    parts = []
    for w in range(worlds):
        part = scenes.tower_world(100 + w, levels, footprint, distance=distance, friction=float(rng.uniform(0.3, 0.8)),
                                  heading=heading, gap=gap)
        part.bodies["mass"][:-1] = rng.uniform(0.5, 2.0, len(part.bodies) - 1).astype(np.float32)
        parts.append(part)
    return scenes.batch(parts)


def settled_trajectory(steps=24, settle=30, speed=4.0, distance=2.2, heading=None, gap=0.0):
    scene = tower_batch(distance=distance, heading=heading, gap=gap)
    world = World(sleep_time=np.inf)
    ids = scene.build(world)
    exported = world.export_scene()
    params = world.step_params(DT)
    oracle = OracleWorld(exported, params)
    for _ in range(settle):
        oracle.step(DT)
    start = oracle.states()
    # launch each world's sphere (the last body of each part, before its plane) toward the tower
    rows = np.sort(exported["owners"][exported["colliders"]["kind"] == R.SHAPE_SPHERE]).astype(np.int64)
    edits = np.zeros(len(rows), R.BODY_EDIT)
    edits["kind"] = R.EDIT_PATCH
    edits["mask"] = R.PATCH_VELOCITY
    for i, row in enumerate(rows):
        direction = -start["position"][row].astype(np.float64)
        direction[1] = 0.0
        v = speed * direction / np.linalg.norm(direction)
        edits["state"]["velocity"][i] = v.astype(np.float32)
        start["velocity"][row] = v.astype(np.float32)
    oracle.edit_bodies(start["body_id"][rows], edits)
    groups = exported["body_world"].astype(np.int64)
    traj = A.FrozenTrajectory(oracle, exported, params, steps, DT, groups, start=start)
    oracle.close()
    world.close()
    return traj, exported, rows


@pytest.fixture(scope="module")
def trajectory():
    """The spheres strike the towers: impacts, contacts forming, clamps switching."""
    return settled_trajectory()


@pytest.fixture(scope="module")
def smooth_trajectory():
    """A contact-smooth regime: the spheres slide and roll toward towers they do not reach; the
    towers rest. No contact forms or breaks and no clamp changes side within a 1e-4 step."""
    return settled_trajectory(steps=16, distance=4.0)


def nominal(traj, exported):
    descs = exported["descs"]
    friction = np.zeros(traj.groups)
    for g in range(traj.groups):
        friction[g] = float(exported["colliders"]["friction"][exported["body_world"][exported["owners"]] == g][0])
    return (descs["inverse_mass"].astype(np.float64), descs["inverse_inertia"].astype(np.float64), friction,
            A.state_vector(traj.start))


def test_the_fp64_forward_follows_the_fp32_trajectory(trajectory):
    traj, exported, rows = trajectory
    im, ii, mu, state = nominal(traj, exported)
    assert traj.counts.min() > 0
    _, final = traj.forward(im, ii, mu, state)
    fp32 = traj.final["position"].astype(np.float64)
    # same contact sets; differences are the fixed-point deltas (2^-18) and FP32 rounding
    assert np.max(np.abs(final[:, :3] - fp32)[traj.dynamic]) < 2e-3
    moved = np.linalg.norm(fp32[rows] - traj.start["position"][rows], axis=1)
    assert np.all(moved > 0.05)  # the spheres travelled


def checked_slots(traj, rows, im, mu, state):
    boxes = [r for r in range(traj.n) if traj.dynamic[r] and r not in rows][:3]
    slots = [traj.inverse_mass_slot(r) for r in boxes] + [traj.friction_slot(0), traj.friction_slot(1)]
    slots += [traj.state_slot(int(rows[0]), 7), traj.state_slot(int(rows[1]), 9)]  # launch velocities
    base = np.concatenate([im, np.zeros(6 * traj.n), mu, state.ravel()])
    return slots, [base[s] for s in slots]


def central_differences(traj, im, ii, mu, state, slots, values, rel):
    base = np.concatenate([im, ii.ravel(), mu, state.ravel()])
    n = traj.n
    out = []
    for s, v in zip(slots, values):
        h = rel * max(abs(v), 1e-3)
        losses = []
        for sign in (1.0, -1.0):
            x = base.copy()
            x[s] += sign * h
            loss, _ = traj.forward(x[:n], x[n:7 * n].reshape(n, 6), x[7 * n:7 * n + traj.groups],
                                   x[7 * n + traj.groups:].reshape(n, 13))
            losses.append(loss)
        out.append((losses[0] - losses[1]) / (2 * h))
    return np.array(out)


def exact_gradient(traj, im, ii, mu, state, slots):
    tangents = np.zeros((len(slots), traj.dim))
    for k, s in enumerate(slots):
        tangents[k, s] = 1.0
    return traj.directional(im, ii, mu, state, tangents)


def test_in_a_contact_smooth_regime_derivatives_match_central_differences(smooth_trajectory):
    traj, exported, rows = smooth_trajectory
    im, ii, mu, state = nominal(traj, exported)
    rng = np.random.default_rng(1)
    traj.target = traj.final["position"].astype(np.float64) + rng.normal(0.0, 0.05, size=(traj.n, 3))
    slots, values = checked_slots(traj, rows, im, mu, state)
    exact = exact_gradient(traj, im, ii, mu, state, slots)
    fd = central_differences(traj, im, ii, mu, state, slots, values, 1e-4)
    # normwise: every component within 1e-3 of the gradient's largest component; the resting boxes'
    # masses move the loss a thousand times less than friction and launch speed do, and their
    # resting contacts sit on the position pass's threshold
    scale = np.max(np.abs(exact))
    assert np.all(np.abs(fd - exact) <= 1e-3 * scale), (fd, exact)
    large = np.abs(exact) >= 0.1 * scale
    assert np.all(np.abs(fd - exact)[large] <= 1e-3 * np.abs(exact)[large]), (fd, exact)


def test_directional_derivatives_match_central_differences(trajectory):
    traj, exported, rows = trajectory
    im, ii, mu, state = nominal(traj, exported)
    rng = np.random.default_rng(0)
    traj.target = traj.final["position"].astype(np.float64) + rng.normal(0.0, 0.05, size=(traj.n, 3))
    boxes = [r for r in range(traj.n) if traj.dynamic[r] and r not in rows][:3]
    slots, values = [], []
    for r in boxes:
        slots.append(traj.inverse_mass_slot(r))
        values.append(im[r])
    slots.append(traj.friction_slot(0))
    values.append(mu[0])
    slots.append(traj.state_slot(int(rows[0]), 7))  # the first sphere's launch velocity, x
    values.append(state[rows[0], 7])
    tangents = np.zeros((len(slots), traj.dim))
    for k, s in enumerate(slots):
        tangents[k, s] = 1.0
    exact = traj.directional(im, ii, mu, state, tangents)
    base = np.concatenate([im, ii.ravel(), mu, state.ravel()])
    n = traj.n

    def central(s, v, rel):
        h = rel * max(abs(v), 1e-3)
        losses = []
        for sign in (1.0, -1.0):
            x = base.copy()
            x[s] += sign * h
            loss, _ = traj.forward(x[:n], x[n:7 * n].reshape(n, 6), x[7 * n:7 * n + traj.groups],
                                   x[7 * n + traj.groups:].reshape(n, 13))
            losses.append(loss)
        return (losses[0] - losses[1]) / (2 * h)

    # h = 1e-4 relative: within 1e-3 of the largest gradient component. The solve's clamps (normal
    # impulse >= 0, the friction cone) are kinks; a difference step that straddles one averages the
    # slopes on both sides, which is what a small component can show.
    # With impacts the loss is only piecewise smooth: contacts form during the trajectory and the
    # solve's clamps change side, so a 1e-4 step straddles kinks. A step small enough to stay
    # between them converges to the forward-mode derivative: every component within 1e-3.
    fd_fine = np.array([central(s, v, 1e-7) for s, v in zip(slots, values)])
    assert np.all(np.abs(fd_fine - exact) <= 1e-3 * np.abs(exact) + 1e-12), (fd_fine, exact)
