"""The kept grid runs on the oracle: the reference's grid derivation behaviours, restated.

The grid index keeps the entries of immovable colliders and of resting (movable, asleep) colliders
sorted across steps and emits them again only when the run changes: a member joins or leaves, a
member's box moves, or the grid resolution moves (grid_resting_{gate,entries,commit}.wgsl, the
`Resting` and `Immovable` derivations of crates/dynamis-world/src/backend/mod.rs:27-112).
  * a resting world owes the grid nothing, however long it rests
        crates/dynamis-world/tests/suite/derivation.rs:128-146
  * editing a sleeping body's pose derives the resting entries on that step     derivation.rs:170-186
  * the first step derives both runs; waking a body derives the resting run it leaves and leaves
    the immovable run alone; moving a static body derives the immovable run
The reference also derives the resting run once its region is 64 steps old (REGION_LIFETIME, for
device counters it cannot otherwise vouch for); the library checks every member every step, so it
has no such lifetime, and a resting world never derives (the reference's own idle-world test asks
the same). The GPU runs are compared with the oracle, counter by counter, in test_gpu_grid_runs.py.
"""
from dynamis_b200 import records as R
from oracle import oracle as O
from test_resting import DT, ground, make, rest_scene, settle_until_asleep, wake


def counter(o, name):
    return int(o.counters()[R.COUNTER[name]])


def settled():
    w, ids = rest_scene()
    o = O.oracle_from_world(w, DT)
    o.step(DT)
    first = {name: counter(o, name) for name in ("IMMOVABLE_EMITTED", "IMMOVABLE_ENTRIES", "RESTING_REBUILD")}
    assert settle_until_asleep(o) < 400
    return w, ids, o, first


def test_the_first_step_derives_both_runs():
    _, _, _, first = settled()
    assert first["IMMOVABLE_EMITTED"] == first["IMMOVABLE_ENTRIES"] > 0
    assert first["RESTING_REBUILD"] == 1


def test_a_resting_world_owes_the_grid_nothing():
    _, ids, o, _ = settled()
    o.step(DT)
    resting = counter(o, "RESTING_ENTRIES")
    assert resting >= len(ids) - 1 and counter(o, "RESTING_LEVELS") != 0
    for _ in range(128):
        o.step(DT)
        assert counter(o, "RESTING_REBUILD") == 0 and counter(o, "RESTING_SORT") == 0
        assert counter(o, "IMMOVABLE_EMITTED") == 0
        assert counter(o, "ENTRIES") == 0 and counter(o, "GRID_LEVELS") == 0
        assert counter(o, "RESTING_ENTRIES") == resting


def test_an_edited_sleeping_body_derives_the_resting_run():
    _, ids, o, _ = settled()
    o.step(DT)
    o.edit_bodies([int(ids[1])], R.body_edit(R.EDIT_PATCH, R.PATCH_POSITION, position=(3.0, 0.4, 0.0)))
    o.step(DT)
    assert counter(o, "RESTING_REBUILD") == 1
    assert counter(o, "IMMOVABLE_EMITTED") == 0


def test_waking_a_body_derives_the_resting_run_it_leaves():
    _, ids, o, _ = settled()
    o.step(DT)
    before = counter(o, "RESTING_ENTRIES")
    wake(o, ids[1])
    o.step(DT)
    assert counter(o, "RESTING_REBUILD") == 1
    assert counter(o, "RESTING_SORT") == counter(o, "RESTING_ENTRIES") < before
    assert counter(o, "ENTRIES") > 0
    assert counter(o, "IMMOVABLE_EMITTED") == 0


def test_moving_a_static_body_derives_the_immovable_run():
    w, ids = make([ground(20.0), dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 0.5, 0))])
    o = O.oracle_from_world(w, DT)
    assert settle_until_asleep(o, 240) < 240
    o.step(DT)
    assert counter(o, "IMMOVABLE_EMITTED") == 0
    o.edit_bodies([int(ids[0])], R.body_edit(R.EDIT_PATCH, R.PATCH_POSITION, position=(0.0, -0.6, 0.0)))
    o.step(DT)
    assert counter(o, "IMMOVABLE_EMITTED") == counter(o, "IMMOVABLE_ENTRIES") > 0


def test_the_resting_field_falls_asleep_into_one_kept_run():
    # scenes.resting_field, the bench's resting world, at 8 x 8 boxes: no box touches another, so
    # every box sleeps within a second and then sits in the resting run, which no step derives again
    from dynamis_b200 import World, scenes

    w = World()
    scenes.resting_field(8).build(w)
    o = O.oracle_from_world(w, DT)
    assert settle_until_asleep(o, 120) < 120
    o.step(DT)
    assert counter(o, "PAIRS") == 0  # asleep against a static plane: no candidate pair
    for _ in range(10):
        o.step(DT)
        assert counter(o, "ENTRIES") == 0 and counter(o, "RESTING_REBUILD") == 0
    assert counter(o, "RESTING_ENTRIES") >= 64 and counter(o, "IMMOVABLE_EMITTED") == 0
