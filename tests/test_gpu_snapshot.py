"""World::snapshot / World::restore on the GPU (dyn_snapshot_take, dyn_snapshot_restore).

As crates/dynamis-world/tests/suite/snapshot.rs:169-197 asks of the reference, a restored world
reproduces the frames it was captured from, bit for bit: here for a forming mixed pile (archived
contacts and warm starts), a sleeping stack (frozen contacts), hanging chains (the joints' runtime)
and a world with queued body commands. A snapshot outlives later steps and restores more than
once; it is refused after the scene changes.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from dynamis_b200 import records as R
from dynamis_b200._native import DynamisError
from test_resting import ground, make

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def frames(world, steps, dt=DT):
    out = []
    for _ in range(steps):
        world.step(dt)
        out.append(world.read_states().copy())
    return out


def same(a, b):
    for x, y in zip(a, b):
        for name in x.dtype.names:
            assert np.array_equal(x[name], y[name]), name


@pytest.mark.parametrize("scene,dt,before,after", [
    (lambda: scenes.random_mix(60, seed=3), DT, 12, 20),
    (lambda: scenes.hanging_chains(3, 2, 8), 1.0 / 120.0, 10, 20),
])
def test_a_restored_world_reproduces_the_frames_it_was_captured_from(scene, dt, before, after):
    w = World()
    scene().build(w)
    frames(w, before, dt)
    snap = w.snapshot()
    counters = w.measured().copy()
    first = frames(w, after, dt)
    w.restore(snap)
    second = frames(w, after, dt)
    same(first, second)
    w.restore(snap)  # a snapshot restores more than once
    same(first, frames(w, after, dt))
    assert w.measured()[R.COUNTER["STEP"]] == counters[R.COUNTER["STEP"]] + after
    snap.close()
    w.close()


def test_frozen_contacts_and_queued_commands_come_back():
    specs = [ground()] + [dict(shape=R.SHAPE_CUBOID, half_extents=(0.4, 0.4, 0.4), position=(0, 0.4 + 0.8 * k, 0),
                               friction=0.6) for k in range(3)]
    w, ids = make(specs)
    for _ in range(400):
        w.step(DT)
        if w.measured()[R.COUNTER["ACTIVE"]] == 0:
            break
    frozen = w.debug_resting()
    assert len(frozen) >= 3
    w.edit_bodies([int(ids[1])], R.body_edit(R.EDIT_WAKE))  # queued before the snapshot
    snap = w.snapshot()
    first = frames(w, 30)
    w.restore(snap)
    assert np.array_equal(np.sort(w.debug_resting(), axis=0), np.sort(frozen, axis=0))
    same(first, frames(w, 30))
    snap.close()
    w.close()


def test_a_snapshot_is_refused_after_the_scene_changes():
    w = World()
    ids = scenes.random_mix(20, seed=2).build(w)
    frames(w, 3)
    snap = w.snapshot()
    w.remove_bodies([int(ids[0])])
    frames(w, 1)
    with pytest.raises(DynamisError):
        w.restore(snap)
    snap.close()
    w.close()
