"""Frozen contacts on the oracle: the reference's sleeping-island behaviours, restated.

When a step ends with both bodies of a contact at rest, the contact is frozen
(freeze_contacts.wgsl); frozen contacts keep their bodies in one island while they sleep
(island_link_resting.wgsl) and are released once either body moves again (thaw_contacts.wgsl).
  * waking one member wakes the resting island it belongs to   crates/dynamis-world/tests/suite/waking.rs:133-153
  * a coupled body wakes when its support leaves                waking.rs:349-380
  * a resting island keeps every member asleep together         waking.rs:216-241
  * resting contacts survive sleep and recycle their slots      activity.rs:111-148
  * a moved static collider releases the sleeping body it held  dependency.rs:43-60
plus the store's own rules (a static row's wake flag lasts one step, static_wake_clear.wgsl). The
GPU path is compared with the oracle in test_gpu_resting.py.
"""
import numpy as np

from dynamis_b200 import World
from dynamis_b200 import records as R
from oracle import oracle as O

DT = 1.0 / 60.0
GRAVITY = {"damping": 0.0, "angular_damping": 0.0}


def make(bodies):
    w = World(**GRAVITY)
    n = len(bodies)
    b = R.body_defaults(n)
    c = R.collider_defaults(n)
    for i, spec in enumerate(bodies):
        spec = dict(spec)
        b["position"][i] = spec.pop("position", (0, 0, 0))
        for key in ("mass", "density", "velocity", "angular_velocity", "orientation"):
            if key in spec:
                b[key][i] = spec.pop(key)
        for key, value in spec.items():
            c[key][i] = value
    ids = w.spawn(b, c)
    return w, ids


def ground(half=5.0):
    return dict(shape=R.SHAPE_CUBOID, half_extents=(half, 0.5, half), mass=0.0, position=(0, -0.5, 0))


def state(o, body_id):
    s = o.states()
    return s[s["body_id"] == body_id][0]


def settle_until_asleep(o, limit=400):
    for step in range(limit):
        o.step(DT)
        if o.counters()[R.COUNTER["ACTIVE"]] == 0:
            return step + 1
    return limit


def wake(o, body_id):
    o.edit_bodies([int(body_id)], R.body_edit(R.EDIT_WAKE))


def test_waking_one_member_wakes_the_resting_island():
    w, ids = make([ground(), dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 0.5, 0)),
                   dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 1.5, 0))])
    o = O.oracle_from_world(w, DT)
    assert settle_until_asleep(o) < 400
    assert state(o, ids[1])["sleeping"] and state(o, ids[2])["sleeping"]
    wake(o, ids[1])
    o.step(DT)
    assert not state(o, ids[2])["sleeping"]


def test_a_stack_wakes_as_one_island_in_one_step():
    # three boxes: the top one touches only the middle one, so only the frozen contacts can reach it
    specs = [ground()] + [dict(shape=R.SHAPE_CUBOID, half_extents=(0.4, 0.4, 0.4), position=(0, 0.4 + 0.8 * k, 0),
                               friction=0.6) for k in range(3)]
    w, ids = make(specs)
    o = O.oracle_from_world(w, DT)
    assert settle_until_asleep(o) < 400
    frozen = o.resting()
    assert len(frozen) >= 3  # ground-box, box-box, box-box
    wake(o, ids[1])
    o.step(DT)
    assert all(not state(o, i)["sleeping"] for i in ids[1:])
    assert o.counters()[R.COUNTER["WOKE"]] == 3


def test_a_coupled_body_wakes_when_its_support_leaves():
    w, ids = make([ground(), dict(shape=R.SHAPE_SPHERE, radius=0.3, position=(-0.5, 1.0, 0)),
                   dict(shape=R.SHAPE_SPHERE, radius=0.3, position=(0.5, 1.0, 0)),
                   dict(shape=R.SHAPE_CUBOID, half_extents=(1.2, 0.25, 1.0), position=(0, 0.25, 0), mass=4.0,
                        friction=0.9)])
    o = O.oracle_from_world(w, DT)
    assert settle_until_asleep(o) < 400
    assert state(o, ids[1])["sleeping"] and state(o, ids[2])["sleeping"]
    o.edit_bodies([int(ids[3])], R.body_edit(R.EDIT_PATCH, R.PATCH_POSITION, position=(50.0, 0.25, 0.0)))
    for _ in range(120):
        o.step(DT)
    assert state(o, ids[1])["position"][1] < 0.5
    assert state(o, ids[2])["position"][1] < 0.5


def test_a_resting_island_keeps_every_member_asleep_together():
    specs = [ground()] + [dict(shape=R.SHAPE_CUBOID, half_extents=(0.4, 0.4, 0.4), position=(0, 0.4 + 0.8 * k, 0),
                               friction=0.6) for k in range(3)]
    w, ids = make(specs)
    o = O.oracle_from_world(w, DT)
    assert settle_until_asleep(o) < 400
    for _ in range(120):
        o.step(DT)
        assert all(state(o, i)["sleeping"] for i in ids[1:])


def rest_scene():
    specs = [ground()]
    for index in range(16):
        x = (index % 4) * 0.85 - 1.3
        z = (index // 4) * 0.85 - 1.3
        specs.append(dict(shape=R.SHAPE_SPHERE, radius=0.4, position=(x, 0.4, z), friction=0.6))
    return make(specs)


def test_resting_contacts_survive_sleep_and_recycle_their_slots():
    w, ids = rest_scene()
    o = O.oracle_from_world(w, DT)
    assert settle_until_asleep(o) < 400
    resting = int(o.counters()[R.COUNTER["RESTING"]])
    assert resting > 0 and len(o.resting()) == resting
    assert o.counters()[R.COUNTER["PAIRS"]] == 0 and o.counters()[R.COUNTER["CONTACTS"]] == 0
    wake(o, ids[1])
    o.step(DT)
    assert o.counters()[R.COUNTER["WOKE"]] > 0 and o.counters()[R.COUNTER["PAIRS"]] > 0
    for _ in range(3):
        o.edit_bodies([int(i) for i in ids[1:]], np.concatenate([R.body_edit(R.EDIT_WAKE)] * 16))
        settle_until_asleep(o)
    assert o.counters()[R.COUNTER["RESTING"]] <= resting + 16


def test_a_moved_static_collider_releases_the_sleeping_body_it_held():
    # the floor is teleported away under a sleeping sphere: its frozen contact carries the floor's
    # wake flag to the sphere, which falls
    w, ids = make([dict(shape=R.SHAPE_CUBOID, half_extents=(20.0, 0.5, 20.0), mass=0.0, position=(0, -0.5, 0)),
                   dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 0.5, 0))])
    o = O.oracle_from_world(w, DT)
    assert settle_until_asleep(o, 240) < 240
    resting = state(o, ids[1])["position"].copy()
    o.edit_bodies([int(ids[0])], R.body_edit(R.EDIT_PATCH, R.PATCH_POSITION, position=(0.0, -20.5, 0.0)))
    for _ in range(30):
        o.step(DT)
    assert state(o, ids[1])["position"][1] < resting[1] - 0.5


def test_a_static_wake_flag_lasts_one_step():
    # a static body teleported next to a sleeping sphere wakes it once; a step later the static row
    # no longer carries a wake flag, so a second sleeping sphere it touches only through the first
    # stays asleep unless the first one moves
    w, ids = make([dict(shape=R.SHAPE_CUBOID, half_extents=(20.0, 0.5, 20.0), mass=0.0, position=(0, -0.5, 0)),
                   dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 0.5, 0))])
    o = O.oracle_from_world(w, DT)
    assert settle_until_asleep(o, 240) < 240
    # a no-op teleport of the floor: its wake flag wakes the sphere resting on it, for one step
    o.edit_bodies([int(ids[0])], R.body_edit(R.EDIT_PATCH, R.PATCH_POSITION, position=(0.0, -0.5, 0.0)))
    o.step(DT)
    assert not state(o, ids[1])["sleeping"]
    assert settle_until_asleep(o, 240) < 240
