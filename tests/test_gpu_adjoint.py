"""World::step_backward on the B200 against the FP64 reference gradient.

Small tower worlds (sleeping off), settled, are struck by spheres launched by a PATCH edit; the
device records the trajectory (dyn_tape_begin, checkpoints every 10 steps) and reverses it
(dyn_backward, which replays each segment from its checkpoint with the narrowphase recomputed).
The FP32 oracle runs the same steps in lockstep (bit-exact with the device); its frozen contact sets
feed the FP64 reference (oracle/adjoint64.cpp). The loss is the summed squared distance of the final
positions to a target.

Two checks:
* along the recorded run: the reference's forward-mode derivatives taken at the recorded FP32 values
  with the recorded branches, which is the linearisation the device adjoint transposes; the device
  gradient must agree to 1e-3 of each kind's largest component, impacts included;
* in a contact-smooth regime (no contact on the friction cone's square-root branch point, none
  changing side of a clamp within the difference step): FP64 central differences of the frozen
  step with h = 1e-4 relative, for per-body mass, per-world friction and the launch velocity.
Orientation gradients are compared in the tangent space of the unit quaternion.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dynamis_b200 import World, records as R, scenes
from oracle import adjoint as A
from oracle.oracle import OracleWorld

from test_adjoint_reference import tower_batch

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0


def record(scene, steps, settle=0, speed=4.0, interval=10, **config):
    """Steps `scene` on the device and on the oracle in lockstep, launches every sphere toward the
    origin, records `steps` steps, reverses them; returns what the checks need."""
    world = World(sleep_time=np.inf, **config)
    scene.build(world)
    exported = world.export_scene()
    params = world.step_params(DT)
    oracle = OracleWorld(exported, params)
    for _ in range(settle):
        world.step(DT)
        oracle.step(DT)
    world.wait()
    start = oracle.states()
    gpu = world.read_states()
    for f in ("position", "orientation", "velocity", "angular_velocity"):
        assert np.array_equal(gpu[f], start[f]), f
    rows = np.sort(exported["owners"][exported["colliders"]["kind"] == R.SHAPE_SPHERE]).astype(np.int64)
    rows = rows[rows < int(params["dynamic_count"][0])]
    if speed and len(rows):
        edits = np.zeros(len(rows), R.BODY_EDIT)
        edits["kind"] = R.EDIT_PATCH
        edits["mask"] = R.PATCH_VELOCITY
        for i, row in enumerate(rows):
            direction = -start["position"][row].astype(np.float64)
            direction[1] = 0.0
            edits["state"]["velocity"][i] = (speed * direction / np.linalg.norm(direction)).astype(np.float32)
            start["velocity"][row] = edits["state"]["velocity"][i]
        world.edit_bodies(start["body_id"][rows], edits)
        oracle.edit_bodies(start["body_id"][rows], edits)
    world.tape_begin(interval)
    for _ in range(steps):
        world.step(DT)
    groups = exported["body_world"].astype(np.int64) if "body_world" in exported else np.zeros(len(start), np.int64)
    traj = A.FrozenTrajectory(oracle, exported, params, steps, DT, groups, start=start)
    oracle.close()
    final = world.read_states()
    for f in ("position", "orientation", "velocity", "angular_velocity"):
        assert np.array_equal(final[f], traj.final[f]), f
    rng = np.random.default_rng(11)
    traj.target = final["position"].astype(np.float64) + rng.normal(0.0, 0.05, size=(len(final), 3))
    grad = np.zeros(len(final), R.BODY_GRAD)
    grad["position"][traj.dynamic] = (2.0 * (final["position"].astype(np.float64) - traj.target))[traj.dynamic]
    out = world.step_backward(grad, steps)
    pg = world.param_grads()
    assert world.tape_steps() == (steps, steps)
    world.tape_end()
    assert np.array_equal(world.read_states()["position"], final["position"])  # the recorded end state is back
    world.close()
    return exported, traj, rows, out, pg


def nominal(traj, exported):
    descs = exported["descs"]
    world_of_collider = (exported["body_world"] if "body_world" in exported
                         else np.zeros(len(descs), np.uint32))[exported["owners"]]
    mu = np.array([exported["colliders"]["friction"][world_of_collider == g][0] for g in range(traj.groups)], np.float64)
    return (descs["inverse_mass"].astype(np.float64), descs["inverse_inertia"].astype(np.float64), mu,
            A.state_vector(traj.start), world_of_collider)


def tangent(q, g):
    return g - q * np.dot(q, g)


def along_record_pairs(traj, exported, out, pg):
    """(device, reference, kind) for every parameter and every dynamic row's start state."""
    im, ii, mu, state, world_of_collider = nominal(traj, exported)
    tangents, device, kinds = [], [], []

    def add(vec, value, kind):
        tangents.append(vec)
        device.append(value)
        kinds.append(kind)

    for g in range(traj.groups):
        t = np.zeros(traj.dim)
        t[traj.friction_slot(g)] = 1.0
        add(t, float(pg["friction"][world_of_collider == g].sum()), "friction")
    dynamic = np.nonzero(traj.dynamic)[0]
    for r in dynamic:
        t = np.zeros(traj.dim)
        t[traj.inverse_mass_slot(int(r))] = 1.0
        add(t, float(pg["inverse_mass"][r]), "inverse_mass")
        t = np.zeros(traj.dim)
        for k in range(6):
            t[traj.inverse_inertia_slot(int(r), k)] = ii[r, k]
        add(t, float(pg["inertia_scale"][r]), "inertia_scale")
        for k, (field, kind) in enumerate([("position", "position")] * 3 + [("orientation", "orientation")] * 4
                                          + [("velocity", "velocity")] * 3 + [("angular_velocity", "angular_velocity")] * 3):
            t = np.zeros(traj.dim)
            t[traj.state_slot(int(r), k)] = 1.0
            comp = [0, 1, 2, 0, 1, 2, 3, 0, 1, 2, 0, 1, 2][k]
            add(t, float(out[field][r][comp]), kind)
    traj.along_record = True
    exact = traj.directional(im, ii, mu, state, np.array(tangents))
    traj.along_record = False
    device, kinds = np.array(device), np.array(kinds)
    for r_i, r in enumerate(dynamic):  # orientation gradients in the tangent space
        sel = np.nonzero(kinds == "orientation")[0][4 * r_i:4 * r_i + 4]
        q = state[r, 3:7]
        device[sel] = tangent(q, device[sel])
        exact[sel] = tangent(q, exact[sel])
    return device, exact, kinds


def check(device, exact, kinds, tolerance):
    failures = []
    for kind in np.unique(kinds):
        m = kinds == kind
        scale = np.max(np.abs(exact[m]))
        err = np.max(np.abs(device[m] - exact[m]))
        print(f"{kind:18s} scale {scale:.3e} max err {err:.3e} ({err / max(scale, 1e-30):.2e})")
        if err > tolerance * scale:
            failures.append((kind, device[m], exact[m]))
    assert not failures, failures


def free_flight() -> scenes.Scene:
    """A spinning sphere in flight above a ground plane: integration and advance alone."""
    bodies = R.body_defaults(1)
    bodies["position"] = (0.0, 5.0, 0.0)
    bodies["velocity"] = (3.0, 1.0, 0.5)
    bodies["angular_velocity"] = (1.0, 2.0, 0.5)
    bodies["mass"] = 1.3
    colliders = R.collider_defaults(1)
    colliders["radius"] = 0.5
    return scenes.Scene(*scenes._ground(bodies, colliders, 0.0, 0.6, 0.0), [], "free_flight")


SCENES = {
    "free_flight": free_flight,
    # columns 2 cm apart, spheres launched straight along x: well-conditioned trajectories, so every
    # state component's gradient is defined to far below the tolerance
    "towers_smooth": lambda: tower_batch(distance=4.0, heading=0.0, gap=0.02),  # the spheres do not reach the towers
    "towers_struck": lambda: tower_batch(distance=2.2, heading=0.0, gap=0.02),  # the spheres strike the towers
}


@pytest.mark.parametrize("name,steps,settle,speed", [("free_flight", 6, 0, 0.0), ("towers_smooth", 16, 30, 4.0),
                                                     ("towers_struck", 24, 30, 4.0)])
def test_the_device_gradient_follows_the_fp64_reference_along_the_recorded_run(name, steps, settle, speed):
    exported, traj, rows, out, pg = record(SCENES[name](), steps, settle=settle, speed=speed)
    device, exact, kinds = along_record_pairs(traj, exported, out, pg)
    check(device, exact, kinds, 1e-3)


def test_benchmark_shaped_towers_parameter_and_launch_gradients_follow_the_reference():
    """Towers as the benchmark builds them (columns face to face, headings drawn) struck by the
    spheres: the parameter gradients and the launch velocities' within 1e-3 of the reference along
    the recorded run. (The resting boxes' own pose gradients are not compared here: with faces in
    contact at zero depth they sit on clamp kinks at every scale.)"""
    exported, traj, rows, out, pg = record(tower_batch(distance=2.2), 24, settle=30)
    device, exact, kinds = along_record_pairs(traj, exported, out, pg)
    keep = np.isin(kinds, ["friction", "inverse_mass", "inertia_scale"])
    dynamic = np.nonzero(traj.dynamic)[0]
    velocity_rows = np.repeat(dynamic, 3)
    launch = np.zeros(len(kinds), bool)
    launch[np.nonzero(kinds == "velocity")[0][np.isin(velocity_rows, rows)]] = True
    check(device[keep | launch], exact[keep | launch], kinds[keep | launch], 1e-3)


def test_in_a_contact_smooth_regime_gradients_match_fp64_central_differences():
    """Towers whose columns stand 2 cm apart and spheres launched straight along x toward towers
    they do not reach: per-body mass, per-world friction and launch velocity (horizontal: a
    vertical launch leaves or presses the ground, a kink at zero) within 1e-3 relative of FP64
    central differences with h = 1e-4 relative."""
    exported, traj, rows, out, pg = record(tower_batch(distance=4.0, heading=0.0, gap=0.02), 16, settle=30)
    im, ii, mu, state, world_of_collider = nominal(traj, exported)
    n = traj.n
    base = np.concatenate([im, ii.ravel(), mu, state.ravel()])

    def loss_at(x):
        return traj.forward(x[:n], x[n:7 * n].reshape(n, 6), x[7 * n:7 * n + traj.groups],
                            x[7 * n + traj.groups:].reshape(n, 13))[0]

    def central(perturb, h):
        xp, xm = base.copy(), base.copy()
        perturb(xp, h)
        perturb(xm, -h)
        return (loss_at(xp) - loss_at(xm)) / (2 * h)

    device, fd, names = [], [], []
    for g in range(traj.groups):
        h = 1e-4 * mu[g]

        def p(x, d, g=g):
            x[traj.friction_slot(g)] += d
        device.append(float(pg["friction"][world_of_collider == g].sum()))
        fd.append(central(p, h))
        names.append(f"friction {g}")
    for r in rows:
        for k in (0, 2):
            h = 1e-4 * max(abs(state[r, 7 + k]), 1e-1)

            def p(x, d, r=r, k=k):
                x[traj.state_slot(int(r), 7 + k)] += d
            device.append(float(out["velocity"][r][k]))
            fd.append(central(p, h))
            names.append(f"launch velocity {r}.{k}")
    for r in np.nonzero(traj.dynamic)[0]:
        m = 1.0 / im[r]
        h = 1e-4 * m

        def p(x, d, r=r, m=m):
            scale = m / (m + d)  # inverse mass and inverse inertia both scale with 1 / mass
            x[traj.inverse_mass_slot(int(r))] *= scale
            for k in range(6):
                x[traj.inverse_inertia_slot(int(r), k)] *= scale
        device.append(-(im[r] * pg["inverse_mass"][r] + pg["inertia_scale"][r]) / m)
        fd.append(central(p, h))
        names.append(f"mass {r}")
    device, fd = np.array(device), np.array(fd)
    for name, d, f in zip(names, device, fd):
        print(f"{name:22s} device {d: .6e} fd {f: .6e}")
    scale = np.max(np.abs(fd))
    assert np.all(np.abs(device - fd) <= 1e-3 * scale), "normwise"
    large = np.abs(fd) >= 0.1 * scale
    assert np.all(np.abs(device - fd)[large] <= 1e-3 * np.abs(fd)[large]), "componentwise"
