"""The 262,144-body mixed pile (the benchmark workload) checked at full size on the GPU.

* Determinism at full size (the behaviour crates/dynamis-world/tests/suite/determinism.rs:61-89
  pins on small scenes): two worlds built from the same seed hold bit-identical states after 60
  steps.
* One full-size step against the oracle: a fresh world and the oracle are loaded with the formed
  pile's states and take one step; every product is compared exactly as on the small scenes.
* Size-independent properties of that step: sorted keys ascend, pairs strictly ascend with
  major < minor and overlapping swept AABBs, every contact holds 1-4 points, and island ids are
  idempotent (an island id is its own island id) and never above the body's row.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from dynamis_b200 import records as R
from oracle.oracle import OracleWorld
from test_gpu_parity import DT, compare_step

pytestmark = pytest.mark.gpu

SETUP_STEPS = 60


@pytest.fixture(scope="module")
def formed_pile():
    world = World()
    scenes.WORKLOADS["mixed_pile_262144"]().build(world)
    for _ in range(SETUP_STEPS):
        world.step(DT)
    world.wait()
    states = world.read_states()
    counters = world.measured()
    world.close()
    return states, counters


def test_two_worlds_from_one_seed_stay_bit_identical(formed_pile):
    states, _ = formed_pile
    twin = World()
    scenes.WORKLOADS["mixed_pile_262144"]().build(twin)
    for _ in range(SETUP_STEPS):
        twin.step(DT)
    twin.wait()
    again = twin.read_states()
    twin.close()
    assert states.tobytes() == again.tobytes()


def test_one_full_size_step_matches_the_oracle(formed_pile):
    states, formed_counters = formed_pile
    assert formed_counters[R.COUNTER["CONTACTS"]] > 50_000, "the pile has not formed"
    world = World()
    scenes.WORKLOADS["mixed_pile_262144"]().build(world)
    world.upload_states(states)
    scene = world.export_scene()
    scene["states"] = states
    oracle = OracleWorld(scene, world.step_params(DT))
    world.step(DT)
    oracle.step(DT)
    world.wait()
    compare_step(world, oracle, 0)
    oracle.close()

    keys, _ = world.debug_entries()
    assert np.all(keys[1:] >= keys[:-1])
    major, minor = world.debug_pairs()
    assert np.all(major < minor)
    packed = (major.astype(np.uint64) << np.uint64(32)) | minor.astype(np.uint64)
    assert np.all(packed[1:] > packed[:-1]), "pairs must be sorted and unique"
    boxes = world.debug_aabbs()
    lo, hi = boxes["min"], boxes["max"]
    overlap = np.all((lo[major] <= hi[minor]) & (lo[minor] <= hi[major]), axis=1)
    assert overlap.all(), "every candidate pair's swept AABBs overlap"
    contacts = world.debug_contacts()
    assert 0 < len(contacts) <= len(major)
    assert np.all((contacts["point_count"] >= 1) & (contacts["point_count"] <= 4))
    islands = world.debug_islands()
    assert np.array_equal(islands[islands], islands)
    assert np.all(islands <= np.arange(len(islands)))
    world.close()


def test_worlds_stay_bit_identical_through_the_pair_stream_widening():
    """150 steps: the pile's pair demand passes half the first pair stream and the stream widens on
    both worlds; their states still agree bit for bit, and the last step refused no pair."""
    finals = []
    for _ in range(2):
        w = World()
        scenes.WORKLOADS["mixed_pile_262144"]().build(w)
        first = None
        for step in range(150):
            w.step(DT)
            if step == 0:
                w.wait()
                first = w.stream_capacity()["pairs"]
        w.wait()
        assert w.stream_capacity()["pairs"] > first, "the pile's demand must widen the pair stream"
        assert w.measured()[R.COUNTER["REFUSED_PAIRS"]] == 0
        finals.append(w.read_states().tobytes())
        w.close()
    assert finals[0] == finals[1]
