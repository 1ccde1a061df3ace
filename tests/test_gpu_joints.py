"""Ball joints on the GPU against the oracle, every step, through the C ABI.

Chains, a branching tree, an unanchored chain falling onto a plane, and joints that break under
load. Each step compares every product test_gpu_parity compares (sorted keys, pairs, contacts,
islands, counters, body states) and the constraint runtime stream: accumulated impulses bit for bit,
reactions within the state tolerance, broken flags exactly.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from dynamis_b200 import records as R
from oracle.oracle import oracle_from_world
from test_gpu_parity import close, compare_step
from test_joints import free_chain, tree_scene

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0


def compare_constraints(world, oracle, step):
    g, o = world.read_constraints(), oracle.constraints()
    assert np.array_equal(g["broken"], o["broken"]), f"step {step}: broken flags differ"
    assert np.array_equal(g["accumulated"].view(np.uint32), o["accumulated"].view(np.uint32)), \
        f"step {step}: accumulated joint impulses differ"
    for f in ("linear_first", "angular_first", "linear_second", "angular_second"):
        assert close(g[f], o[f]), f"step {step}: reaction {f} differs"


def run(world, steps, dt=DT):
    oracle = oracle_from_world(world, dt)
    for step in range(steps):
        world.step(dt)
        oracle.step(dt)
        world.wait()
        compare_step(world, oracle, step)
        compare_constraints(world, oracle, step)
    return oracle


def test_hanging_chains_match_the_oracle_every_step():
    w = World()
    scenes.hanging_chains(3, 2, 8).build(w)
    run(w, 90)
    w.close()


def test_a_joint_tree_matches_the_oracle():
    w = World()
    tree_scene().build(w)
    run(w, 60)
    w.close()


def test_a_falling_free_chain_matches_the_oracle_through_its_landing():
    w = World()
    free_chain().build(w)
    run(w, 200)
    w.close()


def test_joints_that_break_under_load_match_the_oracle():
    sc = scenes.hanging_chains(2, 1, 4)
    joints = sc.joints
    sc.joints = None
    w = World()
    ids = sc.build(w)
    rec = np.zeros(len(joints), R.CONSTRAINT_DESCRIPTOR)
    rec["kind"] = R.CONSTRAINT_BALL
    rec["first_body_id"] = ids[joints["first"]]
    rec["second_body_id"] = ids[joints["second"]]
    rec["flags"] = R.CONSTRAINT_DISABLE_COLLISIONS | R.CONSTRAINT_WARM_START | R.CONSTRAINT_HAS_BREAK
    rec["anchor_a"], rec["anchor_b"] = joints["anchor_a"], joints["anchor_b"]
    rec["axis_a"] = (0.0, 1.0, 0.0)
    rec["break_force"] = np.where(np.arange(len(joints)) % 4 == 1, 300.0, 0.0)  # the second joint of each chain
    w.add_constraints(rec)
    oracle = run(w, 40)
    assert oracle.constraints()["broken"].sum() == 2  # both chains lost their second joint
    w.close()


def test_joints_added_after_stepping_take_hold():
    """A world stepped without joints, then given joints: the chains hang from their anchors."""
    from test_joints import anchor_gaps

    sc = scenes.hanging_chains(2, 2, 5, spin=0.0)
    joints = sc.joints
    sc.joints = None
    w = World()
    ids = sc.build(w)
    for _ in range(3):
        w.step(DT)
    w.wait()
    for jt in joints:
        w.add_ball_joint(int(ids[jt["first"]]), int(ids[jt["second"]]), jt["anchor_a"], jt["anchor_b"])
    for _ in range(240):
        w.step(DT)
    w.wait()
    states = w.read_states()
    assert anchor_gaps(w.export_scene(), states).max() < 1e-2
    links = states[:20]  # the dynamic rows: 4 chains of 5 links
    assert links["position"][:, 1].min() > -3.0  # hanging, not fallen to the ground at -10
    assert w.read_constraints()["broken"].sum() == 0
    w.close()
