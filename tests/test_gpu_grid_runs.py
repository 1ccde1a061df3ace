"""The kept grid runs on the GPU (k_entry_count, k_grid_gate, k_entry_emit, k_entry_merge) against
the oracle, every step from the first.

Each step compares the full parity set (sorted cell keys and entry infos, which the merge of the
three runs must give exactly as one sort of every entry would; pairs, contacts, islands, states)
and the counters of what the step derived again: IMMOVABLE_EMITTED, RESTING_REBUILD, RESTING_SORT,
RESTING_ENTRIES, RESTING_LEVELS. The scenes are those of test_grid_runs.py (a pile of spheres that
falls asleep, is woken and edited; a static floor moved under a sleeping sphere) and a random mix
whose bodies fall asleep at different steps. A query between steps builds its own grid and leaves
the kept runs and the counters alone.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from dynamis_b200 import records as R
from oracle.oracle import oracle_from_world
from test_gpu_parity import compare_step
from test_resting import DT, ground, make, rest_scene

pytestmark = pytest.mark.gpu

RUN_COUNTERS = ["IMMOVABLE_EMITTED", "IMMOVABLE_ENTRIES", "RESTING_REBUILD", "RESTING_SORT", "RESTING_ENTRIES",
                "RESTING_LEVELS", "ENTRIES", "GRID_LEVELS"]


def lockstep(world, oracle, steps, log):
    for _ in range(steps):
        world.step(DT)
        oracle.step(DT)
        world.wait()
        step = len(log)
        compare_step(world, oracle, step)
        gm, om = world.measured(), oracle.counters()
        for name in RUN_COUNTERS:
            assert gm[R.COUNTER[name]] == om[R.COUNTER[name]], f"step {step}: counter {name}"
        log.append({name: int(gm[R.COUNTER[name]]) for name in RUN_COUNTERS} | {"ACTIVE": int(gm[R.COUNTER["ACTIVE"]])})


def both(world, oracle, body_id, edit):
    world.edit_bodies([int(body_id)], edit)
    oracle.edit_bodies([int(body_id)], edit)


def test_a_pile_that_sleeps_wakes_and_is_edited_keeps_its_runs_in_step_with_the_oracle():
    w, ids = rest_scene()
    o = oracle_from_world(w, DT)
    log = []
    lockstep(w, o, 1, log)
    assert log[0]["RESTING_REBUILD"] == 1 and log[0]["IMMOVABLE_EMITTED"] > 0
    while log[-1]["ACTIVE"] != 0 and len(log) < 400:
        lockstep(w, o, 1, log)
    assert log[-1]["ACTIVE"] == 0
    quiet = len(log)
    lockstep(w, o, 40, log)
    assert all(r["RESTING_REBUILD"] == 0 and r["IMMOVABLE_EMITTED"] == 0 for r in log[quiet:])
    assert log[-1]["RESTING_ENTRIES"] > 0 and log[-1]["ENTRIES"] == 0
    both(w, o, ids[1], R.body_edit(R.EDIT_WAKE))
    lockstep(w, o, 1, log)
    assert log[-1]["RESTING_REBUILD"] == 1 and log[-1]["ENTRIES"] > 0
    lockstep(w, o, 60, log)
    both(w, o, ids[5], R.body_edit(R.EDIT_PATCH, R.PATCH_POSITION, position=(3.0, 0.4, 0.0)))
    lockstep(w, o, 30, log)
    o.close()
    w.close()


def test_a_static_floor_moved_under_a_sleeping_sphere_derives_the_immovable_run():
    w, ids = make([ground(20.0), dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 0.5, 0))])
    o = oracle_from_world(w, DT)
    log = []
    while not log or (log[-1]["ACTIVE"] != 0 and len(log) < 240):
        lockstep(w, o, 1, log)
    lockstep(w, o, 5, log)
    assert log[-1]["IMMOVABLE_EMITTED"] == 0
    both(w, o, ids[0], R.body_edit(R.EDIT_PATCH, R.PATCH_POSITION, position=(0.0, -20.5, 0.0)))
    lockstep(w, o, 1, log)
    assert log[-1]["IMMOVABLE_EMITTED"] > 0
    lockstep(w, o, 30, log)
    o.close()
    w.close()


def test_a_random_mix_falling_asleep_body_by_body_matches_the_oracle():
    w = World()
    scenes.random_mix(60, seed=21).build(w)
    o = oracle_from_world(w, DT)
    log = []
    lockstep(w, o, 240, log)
    assert any(r["RESTING_ENTRIES"] > 0 for r in log)
    o.close()
    w.close()


def test_a_query_between_steps_leaves_the_runs_and_counters_alone():
    w, ids = rest_scene()
    o = oracle_from_world(w, DT)
    log = []
    while not log or (log[-1]["ACTIVE"] != 0 and len(log) < 400):
        lockstep(w, o, 1, log)
    lockstep(w, o, 2, log)
    before = w.measured().copy()
    q = np.concatenate([R.ray_query((0.0, 5.0, 0.0), (0.0, -1.0, 0.0), 20.0, R.query_filter(max_hits=8)),
                        R.sphere_query((0.5, 0.4, 0.5), 1.0, R.query_filter(max_hits=8))])
    gq, gh = w.query(q)
    oq, oh = o.query(q)
    assert np.array_equal(gq["count"], oq["count"]) and gq["count"].min() > 0
    assert np.array_equal(gh["scene_target"], oh["scene_target"])
    assert np.array_equal(w.measured(), before)
    lockstep(w, o, 3, log)
    assert all(r["RESTING_REBUILD"] == 0 and r["IMMOVABLE_EMITTED"] == 0 for r in log[-3:])
    o.close()
    w.close()
