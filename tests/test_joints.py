"""Ball joints on the CPU: the solve-order planner, the oracle's joint passes, and the boundary.

The planner restates crates/dynamis-world/src/schedule.rs:105-296 twice, in the product
(dynamis_b200/csrc/scene.cpp, read through dyn_joint_plan) and in the oracle; both must give the
same rows, layers and components. The oracle's joint solve is pinned on behaviours: a hanging chain
keeps its joints together and hangs straight down at rest, jointed neighbours never collide, and
the joint counter counts the filtered pairs.
"""
import numpy as np
import pytest

from dynamis_b200 import DynamisError, World, scenes
from dynamis_b200 import records as R
from oracle.oracle import oracle_from_world

DT = 1.0 / 120.0


def tree_scene():
    """A static anchor holding one box, which holds three boxes, each holding one more box (one
    component). Joints that share a body never share a layer; disjoint ones do."""
    n = 7
    bodies = R.body_defaults(n + 1)
    bodies["density"] = 1000.0
    bodies["mass"][n] = 0.0
    offsets = np.array([[0, -0.5, 0], [-0.6, -1.2, 0], [0, -1.2, 0], [0.6, -1.2, 0],
                        [-0.6, -1.9, 0], [0, -1.9, 0], [0.6, -1.9, 0], [0, 0, 0]], np.float32)
    bodies["position"] = offsets + np.array([0, 5, 0], np.float32)
    colliders = R.collider_defaults(n + 1)
    colliders["shape"][:n] = R.SHAPE_CUBOID
    colliders["half_extents"][:n] = (0.1, 0.25, 0.1)
    colliders["radius"][n] = 0.05
    joints = np.zeros(n, scenes.JOINT)
    pairs = [(7, 0, (0, 0, 0), (0, 0.25, 0)), (0, 1, (-0.1, -0.25, 0), (0, 0.25, 0)), (0, 2, (0, -0.25, 0), (0, 0.25, 0)),
             (0, 3, (0.1, -0.25, 0), (0, 0.25, 0)), (1, 4, (0, -0.25, 0), (0, 0.25, 0)),
             (2, 5, (0, -0.25, 0), (0, 0.25, 0)), (3, 6, (0, -0.25, 0), (0, 0.25, 0))]
    for i, (a, b, pa, pb) in enumerate(pairs):
        joints[i] = (a, b, pa, pb)
    return scenes.Scene(bodies, colliders, [], "tree", joints)


def free_chain(links=6):
    """A chain with no static anchor, falling onto a plane: the planner starts from its head."""
    sc = scenes.hanging_chains(1, 1, links)
    keep = np.arange(links)  # drop the static anchor and its joint; re-add the ground
    bodies, colliders = sc.bodies[keep].copy(), sc.colliders[keep].copy()
    bodies["position"][:, 1] += 6.0
    bodies, colliders = scenes._ground(bodies, colliders, 0.0)
    joints = sc.joints[1:].copy()
    return scenes.Scene(bodies, colliders, [], "free_chain", joints)


def world_of(scene):
    w = World()
    scene.build(w)
    return w


def anchor_gaps(world_scene, states):
    d, rows = world_scene["constraint_descs"], world_scene["constraint_rows"]

    def rotate(q, v):
        u, s = q[:3].astype(np.float64), float(q[3])
        return v + 2.0 * np.cross(u, np.cross(u, v) + s * v)

    gaps = []
    for j in range(len(d)):
        a, b = states[rows[j]["first_row"]], states[rows[j]["second_row"]]
        pa = a["position"] + rotate(a["orientation"], d[j]["anchor_a"].astype(np.float64))
        pb = b["position"] + rotate(b["orientation"], d[j]["anchor_b"].astype(np.float64))
        gaps.append(np.linalg.norm(pa - pb))
    return np.array(gaps)


@pytest.mark.parametrize("make", [lambda: scenes.hanging_chains(3, 2, 5), tree_scene, free_chain])
def test_product_and_oracle_plan_the_same_solve_order(make):
    w = world_of(make())
    plan = w.joint_plan()
    oracle_plan = oracle_from_world(w, DT).joint_plan()
    for key in ("rows", "layers", "components"):
        assert np.array_equal(plan[key], oracle_plan[key]), key
    w.close()


def test_a_chain_is_one_joint_per_layer_from_its_anchor():
    w = world_of(scenes.hanging_chains(2, 1, 5))
    plan = w.joint_plan()
    assert len(plan["components"]) == 2
    assert np.all(plan["layers"][:, 1] == 1)
    # joints are numbered from the anchor down each chain: the layers walk them in that order
    first_component = plan["rows"][:5]
    assert sorted(first_component) == list(first_component)
    w.close()


def test_a_tree_layers_disjoint_joints_together():
    w = world_of(tree_scene())
    plan = w.joint_plan()
    # anchor-box, then the three sibling joints one by one (they share the hub), each grandchild
    # joining the layer after its parent joint
    assert plan["layers"][:, 1].tolist() == [1, 1, 2, 2, 1]
    assert plan["components"].tolist() == [[0, 5]]
    w.close()


def test_a_hanging_chain_holds_together_and_hangs_straight():
    w = world_of(scenes.hanging_chains(1, 1, 6, spin=0.0))
    scene = w.export_scene()
    o = oracle_from_world(w, DT)
    for _ in range(240):
        o.step(DT)
    states = o.states()
    assert anchor_gaps(scene, states).max() < 1e-4
    links = states[:6]
    assert np.all(np.abs(links["position"][:, 0]) < 1e-3) and np.all(np.abs(links["position"][:, 2]) < 1e-3)
    assert np.allclose(links["position"][:, 1], -0.25 - 0.5 * np.arange(6), atol=2e-3)
    o.close()
    w.close()


def test_jointed_neighbours_never_collide_and_are_counted():
    w = world_of(scenes.hanging_chains(2, 2, 6))
    o = oracle_from_world(w, DT)
    scene = w.export_scene()
    rows = scene["constraint_rows"]
    jointed = {tuple(sorted((r["first_row"], r["second_row"]))) for r in rows}
    owners = scene["owners"]
    for _ in range(30):
        o.step(DT)
        c = o.contacts()
        touching = {tuple(sorted((owners[a], owners[b]))) for a, b in zip(c["a"], c["b"])}
        assert not (touching & jointed)
        assert o.counters()[R.COUNTER["JOINTS"]] == len(rows)
    o.close()
    w.close()


def test_a_free_chain_falls_and_keeps_its_joints():
    """In free fall the joints hold to a fraction of a millimetre; the landing stretches them by
    centimetres at the default 8 velocity and 10 position iterations, and they close again."""
    w = world_of(free_chain())
    scene = w.export_scene()
    o = oracle_from_world(w, DT)
    for _ in range(60):
        o.step(DT)
    assert anchor_gaps(scene, o.states()).max() < 5e-4
    for _ in range(300):
        o.step(DT)
    states = o.states()
    assert anchor_gaps(scene, states).max() < 5e-2
    assert states["position"][:6, 1].max() < 1.0  # came down onto the plane
    o.close()
    w.close()


def test_joints_outside_the_path_are_refused():
    w = world_of(scenes.sphere_row(3))
    with pytest.raises(DynamisError):
        w.add_ball_joint(0, 0, (0, 0, 0), (0, 0, 0))
    with pytest.raises(DynamisError):
        w.add_ball_joint(0, 99, (0, 0, 0), (0, 0, 0))
    rec = np.zeros(2, R.CONSTRAINT_DESCRIPTOR)
    rec["first_body_id"], rec["second_body_id"] = 0, 1
    rec[1]["kind"] = 2  # revolute
    with pytest.raises(DynamisError):
        w.add_constraints(rec)
    assert w.constraint_count() == 0  # all or nothing
    rec[1]["kind"] = R.CONSTRAINT_BALL
    rec[1]["flags"] = 2  # a twist limit
    with pytest.raises(DynamisError):
        w.add_constraints(rec)
    rec[1]["flags"] = R.CONSTRAINT_WARM_START
    assert w.add_constraints(rec) == 0 and w.constraint_count() == 2
    w.close()
