"""The autotuner (dyn_autotune) and the launch shapes it picks (dyn_set_launch_config).

* Launch shapes change no result: a 4,096-body mixed pile stepped 40 times with the contact blocks'
  kernels at 64 and at 256 threads, grid-stride launches capped at 4 blocks per SM and the
  persistent GJK and EPA kernels at other block counts, is bit-identical to the default shapes.
* The tuner leaves the world as it found it: states and counters after dyn_autotune equal those
  before; the choice it keeps is one of its candidates; the world then steps bit-identically to an
  untuned twin.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def pile(steps, **launch):
    w = World()
    scenes.mixed_pile(side=16, seed=1).build(w)
    if launch:
        w.set_launch_config(**launch)
    for _ in range(steps):
        w.step(DT)
    w.wait()
    states = w.read_states()
    w.close()
    return states


def test_launch_shapes_change_no_result():
    base = pile(40)
    for shape in ({"solve_threads": 64}, {"solve_threads": 256, "grid_blocks_per_sm": 4},
                  {"gjk_blocks_per_sm": 2, "epa_blocks_per_sm": 12}):
        assert pile(40, **shape).tobytes() == base.tobytes(), shape


def test_the_tuner_leaves_the_world_as_it_found_it():
    tuned, twin = World(), World()
    for w in (tuned, twin):
        scenes.mixed_pile(side=16, seed=1).build(w)
        for _ in range(30):
            w.step(DT)
        w.wait()
    before, counters = tuned.read_states(), tuned.measured()
    config, ms = tuned.autotune(DT, steps=2)
    assert ms > 0.0
    assert config["solve_threads"] in (64, 128, 256)
    assert config["grid_blocks_per_sm"] in (4, 8, 16, 32)
    assert config["gjk_blocks_per_sm"] in (4, 6, 8, 12) and config["epa_blocks_per_sm"] in (4, 8, 12)
    assert tuned.launch_config() == config
    assert tuned.read_states().tobytes() == before.tobytes()
    assert np.array_equal(tuned.measured(), counters)
    for _ in range(10):
        tuned.step(DT)
        twin.step(DT)
    tuned.wait()
    twin.wait()
    assert tuned.read_states().tobytes() == twin.read_states().tobytes()
    tuned.close()
    twin.close()
