"""The hanging-chains and batched-worlds workloads checked against the oracle at full size.

* 64 x 64 chains of 32 boxes (131,072 ball joints, the joint planner's full packing of 8 chains per
  warp) and 4,096 sub-worlds (about 1.76M bodies, where the 4,096 world ids hashed into the cell keys
  actually collide with each other's cells) are each formed on the GPU; then a fresh world and the
  oracle are loaded with the formed states and take one step, and every product is compared as on
  the small scenes (test_gpu_parity.compare_step), the joints' runtime records too
  (test_gpu_joints.compare_constraints).
* Size-independent properties of that step: pairs strictly ascend and never join two sub-worlds;
  every jointed pair is filtered out of the candidate pairs; island ids are idempotent and no island
  spans two sub-worlds or both ends of a broken link.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from dynamis_b200 import records as R
from oracle.oracle import OracleWorld
from test_gpu_joints import compare_constraints
from test_gpu_parity import compare_step

pytestmark = pytest.mark.gpu

SETUP_STEPS = 60


def formed_then_one_step(scene, dt, check_joints):
    world = World()
    scene.build(world)
    for _ in range(SETUP_STEPS):
        world.step(dt)
    world.wait()
    states = world.read_states()
    world.close()

    fresh = World()
    scene.build(fresh)
    fresh.upload_states(states)
    exported = fresh.export_scene()
    exported["states"] = states
    oracle = OracleWorld(exported, fresh.step_params(dt))
    fresh.step(dt)
    oracle.step(dt)
    fresh.wait()
    compare_step(fresh, oracle, 0)
    if check_joints:
        compare_constraints(fresh, oracle, 0)
    oracle.close()
    return fresh, exported


def test_hanging_chains_at_full_size_match_the_oracle():
    scene = scenes.hanging_chains(64, 64, 32)
    world, exported = formed_then_one_step(scene, 1.0 / 120.0, check_joints=True)
    counters = world.measured()
    assert counters[R.COUNTER["CONTACTS"]] > 0, "the chains must touch by then"
    major, minor = world.debug_pairs()
    packed = (major.astype(np.uint64) << np.uint64(32)) | minor.astype(np.uint64)
    assert np.all(packed[1:] > packed[:-1])
    # ball joints disable collisions between their two bodies: linked boxes overlap as candidate
    # pairs, but no contact joins them
    owners = exported["owners"].astype(np.uint64)
    rows = exported["constraint_rows"]
    assert len(rows) == 64 * 64 * 32
    a = np.minimum(rows["first_row"], rows["second_row"]).astype(np.uint64)
    b = np.maximum(rows["first_row"], rows["second_row"]).astype(np.uint64)
    jointed = (a << np.uint64(32)) | b
    pair_bodies = (np.minimum(owners[major], owners[minor]) << np.uint64(32)) | np.maximum(owners[major], owners[minor])
    assert np.isin(jointed, pair_bodies).any(), "linked boxes must meet as candidate pairs"
    contacts = world.debug_contacts()
    ca, cb = owners[contacts["a"]], owners[contacts["b"]]
    contact_bodies = (np.minimum(ca, cb) << np.uint64(32)) | np.maximum(ca, cb)
    assert not np.isin(jointed, contact_bodies).any(), "a jointed pair made a contact"
    islands = world.debug_islands()
    assert np.array_equal(islands[islands], islands)
    world.close()


def test_batched_worlds_at_full_size_match_the_oracle():
    scene = scenes.batched_worlds(4096)
    world, exported = formed_then_one_step(scene, 1.0 / 60.0, check_joints=False)
    body_world = exported["body_world"]
    owners = exported["owners"]
    assert len(np.unique(body_world)) == 4096
    major, minor = world.debug_pairs()
    assert len(major) > 0
    assert np.all(body_world[owners[major]] == body_world[owners[minor]]), "a candidate pair joins two sub-worlds"
    contacts = world.debug_contacts()
    assert len(contacts) > 0
    islands = world.debug_islands()
    assert np.array_equal(islands[islands], islands)
    rows = len(islands)  # the simulated rows (the planes come after them)
    assert np.all(body_world[islands] == body_world[:rows]), "an island spans two sub-worlds"
    world.close()
