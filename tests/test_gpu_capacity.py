"""The pair stream widens after a spill, on the GPU through the C ABI.

crates/dynamis-world/tests/suite/capacity.rs:142-187: a pile heavier than the streams refuses pairs,
the pair stream widens (crates/dynamis-broadphase/src/capacity.rs:27-80, grown() of
crates/dynamis-domain/src/capacity.rs:15-23: here twice the measured demand, at least twice the
stream) and the step stops refusing within a few steps. Here the declared pair stream is far below the demand;
once it has widened, the steps match the oracle, which has room for every pair.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from dynamis_b200 import records as R
from oracle.oracle import oracle_from_world
from test_gpu_parity import compare_step

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def refused(world):
    return int(world.measured()[R.COUNTER["REFUSED_PAIRS"]])


def test_a_spilling_pile_widens_the_pair_stream_and_stops_refusing():
    w = World(capacity={"pairs": 256})
    scenes.mixed_pile(side=8, seed=3).build(w)
    w.step(DT)
    w.wait()
    assert w.stream_capacity()["pairs"] == 256
    assert refused(w) > 0, "the pile must outgrow the declared pair stream"
    demand = int(w.measured()[R.COUNTER["PAIRS"]])
    held = None
    for step in range(1, 13):
        w.step(DT)
        w.wait()
        if refused(w) == 0:
            held = step
            break
    assert held is not None, "the widened stream must serve the pile within twelve steps"
    widened = w.stream_capacity()["pairs"]
    assert widened >= max(2 * 256, 2 * demand)
    for _ in range(5):
        w.step(DT)
    w.wait()
    assert refused(w) == 0 and w.stream_capacity()["pairs"] == widened, "a served stream does not widen again"
    w.close()


def test_steps_after_the_widening_match_the_oracle():
    """A row of spheres whose boxes overlap but whose surfaces are 3 cm apart (beyond the 2 cm
    margin): the first step refuses pairs that could not make contacts, so both sides still agree;
    the stream widens, and impulses then drive the spheres into one another on both sides."""
    w = World(capacity={"pairs": 64})
    ids = scenes.sphere_row(200, gap=0.03).build(w)
    o = oracle_from_world(w, DT)
    w.step(DT)
    o.step(DT)
    w.wait()
    assert refused(w) > 0 and int(o.counters()[R.COUNTER["REFUSED_PAIRS"]]) == 0
    assert w.measured()[R.COUNTER["CONTACTS"]] == o.counters()[R.COUNTER["CONTACTS"]] == 0
    pushed = np.asarray(ids[::10], np.uint32)
    pushes = np.concatenate([R.body_edit(R.EDIT_IMPULSE, velocity=(3.0 if k % 2 == 0 else -3.0, 0.0, 0.0))
                             for k in range(len(pushed))])
    for step in range(1, 40):
        if step == 2:
            w.edit_bodies(pushed, pushes)
            o.edit_bodies(pushed, pushes)
        w.step(DT)
        o.step(DT)
        w.wait()
        compare_step(w, o, step)
    assert refused(w) == 0 and int(o.counters()[R.COUNTER["CONTACTS"]]) > 0
    o.close()
    w.close()


def test_a_stream_that_serves_the_pile_never_widens():
    w = World()
    scenes.mixed_pile(side=8, seed=3).build(w)
    for _ in range(5):
        w.step(DT)
    w.wait()
    first = w.stream_capacity()["pairs"]
    for _ in range(5):
        w.step(DT)
    w.wait()
    assert refused(w) == 0 and w.stream_capacity()["pairs"] == first
    w.close()
