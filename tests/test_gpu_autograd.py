"""dynamis_b200.autograd.rollout: a torch.autograd.Function over the C ABI's step_backward.

Two tower worlds in the contact-smooth regime (columns 2 cm apart, spheres launched along x toward
towers they do not reach) are rolled out through the Function; loss.backward() must give the
gradients of per-body mass, per-collider friction and starting velocity that FP64 central
differences (h = 1e-4 relative) of the frozen-contact step give, within 1e-3 relative.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dynamis_b200 import World, records as R
from dynamis_b200.autograd import rollout
from oracle import adjoint as A
from oracle.oracle import OracleWorld

from test_adjoint_reference import tower_batch

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0
STEPS = 16


def test_rollout_gradients_match_fp64_central_differences():
    scene = tower_batch(distance=4.0, heading=0.0, gap=0.02)
    world = World(sleep_time=np.inf)
    scene.build(world)
    exported = world.export_scene()
    params = world.step_params(DT)
    oracle = OracleWorld(exported, params)
    for _ in range(30):
        world.step(DT)
        oracle.step(DT)
    start = world.read_states()
    n = len(start)
    descs = exported["descs"]
    mass = np.where(descs["inverse_mass"] > 0, 1.0 / np.maximum(descs["inverse_mass"], 1e-30), 0.0)
    spheres = np.sort(exported["owners"][exported["colliders"]["kind"] == R.SHAPE_SPHERE]).astype(np.int64)
    velocity = start["velocity"].copy()
    velocity[spheres] = (4.0, 0.0, 0.0)
    # the oracle takes the launch as a PATCH edit at its first recorded step, the device as a state upload
    edits = np.zeros(len(spheres), R.BODY_EDIT)
    edits["kind"] = R.EDIT_PATCH
    edits["mask"] = R.PATCH_VELOCITY
    edits["state"]["velocity"] = (4.0, 0.0, 0.0)
    oracle.edit_bodies(start["body_id"][spheres], edits)
    launched = oracle.states()
    launched["velocity"][spheres] = (4.0, 0.0, 0.0)
    traj = A.FrozenTrajectory(oracle, exported, params, STEPS, DT, exported["body_world"].astype(np.int64), start=launched)
    oracle.close()

    t_mass = torch.tensor(mass.astype(np.float32), requires_grad=True)
    t_friction = torch.tensor(exported["colliders"]["friction"].astype(np.float32), requires_grad=True)
    t_velocity = torch.tensor(velocity.astype(np.float32), requires_grad=True)
    final = rollout(world, t_mass, t_friction, t_velocity, STEPS, DT)
    # the same trajectory (the masses pass through 1 / (1 / m), which may move their last bit)
    assert np.allclose(final.detach().numpy(), traj.final["position"], atol=1e-5)
    rng = np.random.default_rng(5)
    target = torch.from_numpy((traj.final["position"] + rng.normal(0.0, 0.05, (n, 3))).astype(np.float32))
    dynamic = torch.from_numpy(traj.dynamic)
    loss = (((final - target) ** 2).sum(dim=1) * dynamic).sum()
    loss.backward()
    world.close()

    traj.target = target.numpy().astype(np.float64)
    im = descs["inverse_mass"].astype(np.float64)
    ii = descs["inverse_inertia"].astype(np.float64)
    world_of_collider = exported["body_world"][exported["owners"]]
    mu = np.array([exported["colliders"]["friction"][world_of_collider == g][0] for g in range(traj.groups)], np.float64)
    state = A.state_vector(traj.start)
    base = np.concatenate([im, ii.ravel(), mu, state.ravel()])

    def loss_at(x):
        return traj.forward(x[:n], x[n:7 * n].reshape(n, 6), x[7 * n:7 * n + traj.groups],
                            x[7 * n + traj.groups:].reshape(n, 13))[0]

    def central(perturb, h):
        xp, xm = base.copy(), base.copy()
        perturb(xp, h)
        perturb(xm, -h)
        return (loss_at(xp) - loss_at(xm)) / (2 * h)

    got, want = [], []
    for r in np.nonzero(traj.dynamic)[0]:
        m = mass[r]

        def p(x, d, r=r, m=m):
            s = m / (m + d)
            x[traj.inverse_mass_slot(int(r))] *= s
            for k in range(6):
                x[traj.inverse_inertia_slot(int(r), k)] *= s
        got.append(float(t_mass.grad[r]))
        want.append(central(p, 1e-4 * m))
    for g in range(traj.groups):
        def p(x, d, g=g):
            x[traj.friction_slot(g)] += d
        got.append(float(t_friction.grad[torch.from_numpy(world_of_collider == g)].sum()))
        want.append(central(p, 1e-4 * mu[g]))
    for r in spheres:
        def p(x, d, r=r):
            x[traj.state_slot(int(r), 7)] += d
        got.append(float(t_velocity.grad[r, 0]))
        want.append(central(p, 1e-4 * 4.0))
    got, want = np.array(got), np.array(want)
    scale = np.max(np.abs(want))
    assert np.all(np.abs(got - want) <= 1e-3 * scale), (got, want)
    large = np.abs(want) >= 0.1 * scale
    assert np.all(np.abs(got - want)[large] <= 1e-3 * np.abs(want)[large]), (got, want)
