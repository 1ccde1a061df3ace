"""Lagged observations on the GPU (World::observe_bodies / try_state, crates/dynamis-world/src/
observation.rs:480-516): after each step the observed records and counters are copied into a ring of
pinned host slots; a read takes the newest completed copy and never waits."""
import numpy as np
import pytest

from dynamis_b200 import DynamisError, World, scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def test_an_observation_of_all_bodies_matches_the_state_after_its_step():
    w = World()
    ids = scenes.random_mix(20, seed=3).build(w)
    w.observe_bodies()
    for _ in range(10):
        w.step(DT)
    w.wait()
    states = {int(s["body_id"]): s for s in w.read_states()}
    for i in ids:
        got = w.try_state(int(i))
        assert got is not None
        rec, step = got
        assert step == 10
        assert rec.tobytes() == states[int(i)].tobytes()
    counters, step = w.try_counters()
    assert step == 10 and np.array_equal(counters, w.measured())
    w.close()


def test_reads_never_run_ahead_of_the_steps_taken():
    w = World()
    ids = scenes.mixed_pile(side=12, seed=4).build(w)
    w.observe_bodies([ids[0], ids[7]])
    seen = []
    for n in range(1, 16):
        w.step(DT)
        got = w.try_state(int(ids[7]))  # no wait: may be an older step, or none yet
        if got is not None:
            seen.append(got[1])
            assert got[1] <= n
    w.wait()
    rec, step = w.try_state(int(ids[7]))
    assert step == 15
    assert seen == sorted(seen)
    with pytest.raises(DynamisError):
        w.try_state(int(ids[3]))  # not observed
    w.close()


def test_a_removed_body_drops_out_of_the_observations():
    w = World()
    ids = scenes.random_mix(12, seed=5).build(w)
    w.observe_bodies()
    w.step(DT)
    w.remove_bodies([ids[2]])
    w.step(DT)
    w.wait()
    assert w.try_state(int(ids[1]))[1] == 2
    with pytest.raises(DynamisError):
        w.try_state(int(ids[2]))
    w.close()
