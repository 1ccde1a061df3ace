"""Frozen contacts on the GPU (rest.cuh: freeze, thaw, island links, static wake clear) against the
oracle, every step.

The scenes of test_resting.py (the reference's sleeping-island behaviours, waking.rs, activity.rs,
dependency.rs) run through the C ABI with the full parity check each step (pairs, contacts,
islands, counters including RESTING and REFUSED_RESTING, body states) plus the set of frozen
contacts (body ids, generations, colliders) compared as a set: the device's store holds them in the
order its appends land in. A removed support (which re-uploads the scene) must still release the
sleeping body it held, as the reference's dependency.rs:127-155 asks.
"""
import numpy as np
import pytest

from dynamis_b200 import records as R
from oracle.oracle import oracle_from_world
from test_gpu_parity import compare_step
from test_resting import DT, ground, make, rest_scene

pytestmark = pytest.mark.gpu


def same_frozen(world, oracle, step):
    g, o = world.debug_resting(), oracle.resting()
    assert len(g) == len(o), f"step {step}: {len(g)} frozen contacts vs {len(o)}"
    g = g[np.lexsort(g.T[::-1])]
    o = o[np.lexsort(o.T[::-1])]
    assert np.array_equal(g, o), f"step {step}: frozen contacts differ"
    gm, om = world.measured(), oracle.counters()
    for name in ("RESTING", "REFUSED_RESTING"):
        assert gm[R.COUNTER[name]] == om[R.COUNTER[name]], f"step {step}: counter {name}"


def lockstep(world, oracle, steps, until_asleep=False):
    for step in range(steps):
        world.step(DT)
        oracle.step(DT)
        world.wait()
        compare_step(world, oracle, step)
        same_frozen(world, oracle, step)
        if until_asleep and oracle.counters()[R.COUNTER["ACTIVE"]] == 0:
            return step + 1
    return steps


def both(world, oracle, body_ids, edit):
    world.edit_bodies([int(i) for i in body_ids], np.concatenate([edit] * len(body_ids)))
    oracle.edit_bodies([int(i) for i in body_ids], np.concatenate([edit] * len(body_ids)))


def gpu_state(world, body_id):
    s = world.read_states()
    return s[s["body_id"] == body_id][0]


def test_a_stack_sleeps_then_wakes_as_one_island():
    specs = [ground()] + [dict(shape=R.SHAPE_CUBOID, half_extents=(0.4, 0.4, 0.4), position=(0, 0.4 + 0.8 * k, 0),
                               friction=0.6) for k in range(3)]
    w, ids = make(specs)
    o = oracle_from_world(w, DT)
    assert lockstep(w, o, 400, until_asleep=True) < 400
    assert len(w.debug_resting()) >= 3
    both(w, o, [ids[1]], R.body_edit(R.EDIT_WAKE))
    lockstep(w, o, 1)
    assert w.measured()[R.COUNTER["WOKE"]] == 3
    lockstep(w, o, 60)
    w.close()


def test_a_coupled_body_wakes_when_its_support_leaves():
    w, ids = make([ground(), dict(shape=R.SHAPE_SPHERE, radius=0.3, position=(-0.5, 1.0, 0)),
                   dict(shape=R.SHAPE_SPHERE, radius=0.3, position=(0.5, 1.0, 0)),
                   dict(shape=R.SHAPE_CUBOID, half_extents=(1.2, 0.25, 1.0), position=(0, 0.25, 0), mass=4.0,
                        friction=0.9)])
    o = oracle_from_world(w, DT)
    assert lockstep(w, o, 400, until_asleep=True) < 400
    both(w, o, [ids[3]], R.body_edit(R.EDIT_PATCH, R.PATCH_POSITION, position=(50.0, 0.25, 0.0)))
    lockstep(w, o, 120)
    assert gpu_state(w, ids[1])["position"][1] < 0.5 and gpu_state(w, ids[2])["position"][1] < 0.5
    w.close()


def test_a_sleeping_pile_recycles_its_frozen_contacts():
    w, ids = rest_scene()
    o = oracle_from_world(w, DT)
    assert lockstep(w, o, 400, until_asleep=True) < 400
    resting = int(w.measured()[R.COUNTER["RESTING"]])
    assert resting > 0 and w.measured()[R.COUNTER["PAIRS"]] == 0
    for _ in range(2):
        both(w, o, ids[1:], R.body_edit(R.EDIT_WAKE))
        lockstep(w, o, 400, until_asleep=True)
    assert w.measured()[R.COUNTER["RESTING"]] <= resting + 16
    w.close()


def test_a_moved_static_collider_releases_the_sleeping_body_it_held():
    w, ids = make([dict(shape=R.SHAPE_CUBOID, half_extents=(20.0, 0.5, 20.0), mass=0.0, position=(0, -0.5, 0)),
                   dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 0.5, 0))])
    o = oracle_from_world(w, DT)
    assert lockstep(w, o, 240, until_asleep=True) < 240
    resting = gpu_state(w, ids[1])["position"].copy()
    both(w, o, [ids[0]], R.body_edit(R.EDIT_PATCH, R.PATCH_POSITION, position=(0.0, -20.5, 0.0)))
    lockstep(w, o, 30)
    assert gpu_state(w, ids[1])["position"][1] < resting[1] - 0.5
    w.close()


def test_a_removed_support_releases_the_sleeping_body_it_held():
    # World::remove re-uploads the scene here; the frozen contacts, kept by body id, carry over, and
    # the one naming the removed box disturbs the sleeping box it held (thaw_contacts.wgsl:49-60)
    w, ids = make([ground(), dict(shape=R.SHAPE_CUBOID, half_extents=(1.0, 0.5, 1.0), position=(0, 0.5, 0)),
                   dict(shape=R.SHAPE_CUBOID, half_extents=(1.0, 0.5, 1.0), position=(0, 1.5, 0))])
    for step in range(900):
        w.step(DT)
        if step % 30 == 29:
            w.wait()
            if w.measured()[R.COUNTER["ACTIVE"]] == 0:
                break
    w.wait()
    assert w.measured()[R.COUNTER["ACTIVE"]] == 0
    resting = gpu_state(w, ids[2])["position"].copy()
    w.remove_bodies([int(ids[1])])
    for _ in range(30):
        w.step(DT)
    w.wait()
    assert gpu_state(w, ids[2])["position"][1] < resting[1] - 0.5
    w.close()
