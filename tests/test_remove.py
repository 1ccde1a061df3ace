"""Body removal on the CPU side of the boundary: World::remove (crates/dynamis-world/src/body.rs:
132-155) refuses an unknown or still-referenced body; a removed body and its colliders leave the
rows, the other bodies keep their ids, and ids are not reused.
"""
import numpy as np
import pytest

from dynamis_b200 import DynamisError, World, scenes
from dynamis_b200 import records as R
from oracle.oracle import oracle_from_world

DT = 1.0 / 60.0


def test_a_removed_body_leaves_the_rows_and_the_others_keep_their_ids():
    w = World()
    ids = scenes.sphere_row(5).build(w)
    before = w.export_scene()
    w.remove_bodies([ids[1], ids[3]])
    after = w.export_scene()
    assert len(after["states"]) == len(before["states"]) - 2
    assert len(after["colliders"]) == len(before["colliders"]) - 2
    kept = sorted(int(i) for i in after["states"]["body_id"])
    assert kept == [int(ids[0]), int(ids[2]), int(ids[4])]
    with pytest.raises(DynamisError):
        w.read_state(int(ids[1]))
    s = w.read_state(int(ids[2]))
    assert np.array_equal(s["position"], before["states"][2]["position"])
    w.close()


def test_removal_refuses_unknown_repeated_and_referenced_bodies():
    w = World()
    ids = scenes.sphere_row(4).build(w)
    with pytest.raises(DynamisError):
        w.remove_bodies([99])
    with pytest.raises(DynamisError):
        w.remove_bodies([ids[0], ids[0]])
    w.add_ball_joint(int(ids[2]), int(ids[3]), (0, 0, 0), (0, 0, 0))
    with pytest.raises(DynamisError):
        w.remove_bodies([ids[3]])
    w.remove_bodies([ids[0]])
    with pytest.raises(DynamisError):
        w.remove_bodies([ids[0]])  # already gone
    with pytest.raises(DynamisError):
        w.apply_impulse(int(ids[0]), (0.0, 1.0, 0.0))
    assert len(w.export_scene()["states"]) == 3
    w.close()


def test_new_bodies_after_a_removal_take_fresh_ids():
    w = World()
    first = scenes.sphere_row(3).build(w)
    w.remove_bodies([first[1]])
    more = scenes.sphere_row(2, height=9.0).build(w)
    assert min(int(i) for i in more) >= 3
    assert len(w.export_scene()["states"]) == 4
    w.close()


def test_the_oracle_steps_the_world_left_after_a_removal():
    w = World()
    ids = scenes.random_mix(16, seed=9).build(w)
    w.remove_bodies(ids[:4])
    o = oracle_from_world(w, DT)
    for _ in range(10):
        o.step(DT)
    s = o.states()
    assert len(s) == len(ids) - 4
    assert not set(int(i) for i in s["body_id"]) & set(int(i) for i in ids[:4])
    assert np.isfinite(s["position"]).all()
    o.close()
    w.close()


def test_observations_are_not_ready_before_a_step():
    w = World()
    ids = scenes.sphere_row(3).build(w)
    assert w.try_state(int(ids[0])) is None
    w.observe_bodies([ids[0], ids[2]])
    assert w.try_state(int(ids[0])) is None and w.try_counters() is None
    with pytest.raises(DynamisError):
        w.observe_bodies([42])
    w.observe_bodies()
    w.stop_observing()
    w.close()
