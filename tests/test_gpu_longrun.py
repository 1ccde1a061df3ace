"""Long runs on the GPU, judged by bounds instead of state by state (they are chaotic).

* The falling-boxes workload (1,000 unit cubes on a 10x10x10 lattice, dt 1/60) for its full 600
  steps, sampled every 10 steps:
  - total energy (kinetic + rotational + gravitational, dynamis_b200.diagnostics) never exceeds its
    starting value: contacts, friction, damping and position correction only take energy out,
    except where a correction lifts a body, which the starting energy bounds too;
  - no body moves faster than free fall from the lattice's top (sqrt(2 g h), h = 10.55 m): a
    contact that injects energy shows first as one body outrunning gravity;
  - the whole pile's mean horizontal velocity stays under 0.25 m/s, 2.5 % of the free-fall speed
    scale sqrt(2 g h): the ground's friction is the only horizontal force, so a solver that pushes
    momentum into the pile shows as a drift of the whole pile;
  - the deepest overlap of any contact point stays under 0.15 m and no cube's centre sinks below
    0.5 - 0.15 m: under the weight of a ten-cube column the position pass (relaxation 0.8, its
    default iterations) leaves the bottom contacts more than the single-body margin deep, and 0.15 m
    bounds that for this pile (measured: 0.116 m at worst over the run);
  - every state stays finite.
* Two of the reference's long-run behaviours (crates/dynamis-world/tests/suite/dynamics.rs):
  a dropped box settles within the contact margin plus slop (:215-240), and a 16-box tower holds
  its spacing within margin + level x slop and does not wander more than 0.2 m (:176-213).
"""
import numpy as np
import pytest

from dynamis_b200 import World, diagnostics, scenes
from dynamis_b200 import records as R

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
G = 9.81


def test_falling_boxes_stay_within_the_long_run_bounds():
    world = World()
    scenes.falling_boxes(seed=0).build(world)
    top = 0.6 + 9 * 1.1 + 0.05
    speed_bound = np.sqrt(2.0 * G * top)
    start = diagnostics.summary(world, DT, stepped=False)["energy"]["total"]
    for step in range(1, 601):
        world.step(DT)
        if step % 10:
            continue
        s = diagnostics.summary(world, DT)
        states = world.read_states()
        assert np.all(np.isfinite(states["position"])) and np.all(np.isfinite(states["velocity"]))
        assert s["energy"]["total"] <= start * (1.0 + 1e-6), f"step {step}: energy rose above its start"
        speed = np.linalg.norm(states["velocity"].astype(np.float64), axis=1).max()
        assert speed <= speed_bound, f"step {step}: a body moves at {speed:.2f} m/s, faster than free fall"
        mean = s["mean_velocity"]
        assert np.hypot(mean[0], mean[2]) <= 0.25, f"step {step}: the pile drifts at {mean}"
        assert s["deepest_penetration"] <= 0.15, f"step {step}: overlap {s['deepest_penetration']:.3f} m"
        dynamic = diagnostics.masses(world.export_scene()["descs"]) > 0
        assert states["position"][dynamic, 1].min() >= 0.5 - 0.15
    world.close()


def box_scene(boxes, ground_half=(40.0, 0.5, 40.0)):
    """Unit boxes (half-extent 0.5 m, mass 1, friction 0.7, restitution 0) at the given positions,
    and a static cuboid ground whose top face is at y = 0."""
    n = len(boxes)
    bodies = R.body_defaults(n + 1)
    bodies["position"][:n] = boxes
    bodies["position"][n] = (0.0, -ground_half[1], 0.0)
    bodies["mass"][n] = 0.0
    colliders = R.collider_defaults(n + 1)
    colliders["shape"] = R.SHAPE_CUBOID
    colliders["half_extents"][:n] = 0.5
    colliders["half_extents"][n] = ground_half
    colliders["friction"] = 0.7
    colliders["restitution"] = 0.0
    return scenes.Scene(bodies, colliders, [], "boxes")


def test_a_dropped_box_settles_within_the_contact_margin():
    margin = 0.02
    world = World(contact_margin=margin)
    ids = box_scene(np.array([[0.0, 2.5, 0.0]])).build(world)
    for _ in range(240):
        world.step(DT)
    state = world.read_state(int(ids[0]))
    overlap = 0.5 - float(state["position"][1])
    slop = float(world.step_params(DT)["slop"][0])
    assert overlap <= margin + slop, f"a landing body sank {overlap:.4f} m"
    world.close()


def test_a_resting_tower_holds_its_spacing():
    levels = 16
    world = World()
    positions = np.array([[0.0, 0.5 + level * 1.0005, 0.0] for level in range(levels)], np.float32)
    ids = box_scene(positions).build(world)
    for _ in range(240):
        world.step(DT)
    params = world.step_params(DT)
    margin, slop = float(params["contact_margin"][0]), float(params["slop"][0])
    for level in range(levels):
        p = world.read_state(int(ids[level]))["position"]
        assert abs(float(p[1]) - (0.5 + level)) <= margin + level * slop, f"level {level} at y = {p[1]}"
        assert abs(float(p[0])) < 0.2 and abs(float(p[2])) < 0.2, f"level {level} wandered to {p}"
    world.close()
