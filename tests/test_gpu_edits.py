"""Body commands on the GPU against the oracle, every step, through the C ABI.

Each step queues a seeded mix of every command kind (patches, forces, forces at a point, torques,
impulses, impulses at a point, angular impulses, sleep, wake; several on one body, on static
bodies too) on both sides, then compares every product test_gpu_parity compares. Steps without
commands follow steps with them: the device must apply each queued command exactly once.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from dynamis_b200 import records as R
from oracle.oracle import oracle_from_world
from test_edits import random_edits
from test_gpu_joints import compare_constraints
from test_gpu_parity import compare_step

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def run(world, ids, steps, per_step, seed, every=1, dt=DT, joints=False):
    rng = np.random.default_rng(seed)
    oracle = oracle_from_world(world, dt)
    for step in range(steps):
        if step % every == 0:
            who, recs = random_edits(rng, ids, per_step)
            world.edit_bodies(who, recs)
            oracle.edit_bodies(who, recs)
        world.step(dt)
        oracle.step(dt)
        world.wait()
        compare_step(world, oracle, step)
        if joints:
            compare_constraints(world, oracle, step)
    oracle.close()


def test_commands_match_the_oracle_every_step():
    w = World()
    ids = scenes.random_mix(24, seed=11).build(w)
    run(w, ids, 40, 10, seed=1)
    w.close()


def test_commands_on_some_steps_only_are_applied_once():
    w = World()
    ids = scenes.random_mix(20, seed=12).build(w)
    run(w, ids, 45, 6, seed=2, every=3)
    w.close()


def test_commands_on_a_lattice_with_sleepers():
    """A settled lattice: most bodies asleep when the commands wake, push and re-freeze them."""
    w = World()
    ids = scenes.box_lattice(64, seed=9).build(w)
    o = oracle_from_world(w, DT)
    for step in range(60):  # settle on both sides
        w.step(DT)
        o.step(DT)
    w.wait()
    compare_step(w, o, 59)
    rng = np.random.default_rng(5)
    for step in range(30):
        who, recs = random_edits(rng, ids, 8)
        w.edit_bodies(who, recs)
        o.edit_bodies(who, recs)
        w.step(DT)
        o.step(DT)
        w.wait()
        compare_step(w, o, 60 + step)
    o.close()
    w.close()


def test_commands_on_jointed_chains():
    w = World()
    ids = scenes.hanging_chains(2, 2, 6).build(w)
    run(w, ids, 40, 6, seed=3, dt=1.0 / 120.0, joints=True)
    w.close()


def test_commands_in_a_batch_of_worlds():
    from test_batch import parts

    w = World()
    ids = scenes.batch(parts()).build(w)
    run(w, ids, 30, 12, seed=4)
    w.close()


def test_many_commands_grow_the_queue():
    """More commands in one step than the first queue holds (256): the queue and the step graph grow."""
    w = World()
    ids = scenes.mixed_pile(side=8, seed=3).build(w)
    run(w, ids, 6, 700, seed=6, every=2)
    w.close()


def test_a_sleep_command_matches_the_oracle_counts():
    w = World()
    ids = scenes.random_mix(12, seed=13).build(w)
    o = oracle_from_world(w, DT)
    sleepers = np.asarray(ids[:4], np.uint32)
    recs = np.concatenate([R.body_edit(R.EDIT_SLEEP)] * 4)
    w.edit_bodies(sleepers, recs)
    o.edit_bodies(sleepers, recs)
    w.step(DT)
    o.step(DT)
    w.wait()
    compare_step(w, o, 0)
    assert w.measured()[R.COUNTER["SLEPT"]] == o.counters()[R.COUNTER["SLEPT"]] >= 1
    o.close()
    w.close()


def test_bodies_removed_after_stepping_match_the_oracle():
    """A pile steps on the GPU, loses some bodies (several of them in contact), and steps on: the
    rest keep their simulated states and match the oracle built from the world after the removal."""
    w = World()
    ids = scenes.random_mix(24, seed=14).build(w)
    for _ in range(20):
        w.step(DT)
    w.wait()
    gone = np.asarray(ids[2:8], np.uint32)
    before = {int(s["body_id"]): s for s in w.read_states()}
    w.remove_bodies(gone)
    o = oracle_from_world(w, DT)
    kept = o.states()
    for s in kept:  # the oracle starts from the GPU's states of the remaining bodies
        assert np.array_equal(s["position"], before[int(s["body_id"])]["position"])
    for step in range(30):
        w.step(DT)
        o.step(DT)
        w.wait()
        compare_step(w, o, step)
    assert not set(int(i) for i in w.read_states()["body_id"]) & set(int(i) for i in gone)
    o.close()
    w.close()


def test_bodies_spawned_after_a_removal_match_the_oracle():
    w = World()
    ids = scenes.random_mix(16, seed=15).build(w)
    for _ in range(10):
        w.step(DT)
    w.remove_bodies(ids[:3])
    scenes.sphere_row(3, height=6.0, gravity=True).build(w)
    o = oracle_from_world(w, DT)
    for step in range(25):
        w.step(DT)
        o.step(DT)
        w.wait()
        compare_step(w, o, step)
    o.close()
    w.close()
