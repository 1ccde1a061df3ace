"""Continuous collision on the oracle: the reference's CCD behaviours, restated.

  * an unflagged bullet tunnels through a small target; a CCD bullet stops at its surface
                                                    crates/dynamis-world/tests/suite/dynamics.rs:241-274
  * a CCD rod is stopped by its leading face and comes to rest against the wall     dynamics.rs:276-308
  * continuous collision keeps a spinning rod out of the wall it sweeps              dynamics.rs:310-357
  * a CCD bullet stops at the nearest obstacle of a chain                            dynamics.rs:359-386
  * clearing the flag restores tunnelling                                            dynamics.rs:693-710
  * a CCD bullet stops at the anchor it may touch                                    filter.rs:145-170
The library's own rule for equal sweep times (the first pair in collider order keeps the impact)
and the set_ccd host checks are tested here too; the GPU path is compared with the oracle in
test_gpu_ccd.py.
"""
import numpy as np
import pytest

from dynamis_b200 import World
from dynamis_b200 import records as R
from dynamis_b200._native import DynamisError
from oracle import oracle as O

DT = 1.0 / 60.0
STATIC = {"gravity": (0.0, 0.0, 0.0), "damping": 0.0, "angular_damping": 0.0}


def make(bodies, config=None):
    """bodies: list of dicts (shape, position, velocity, mass, ccd, collider fields)."""
    w = World(**(config or STATIC))
    n = len(bodies)
    b = R.body_defaults(n)
    c = R.collider_defaults(n)
    for i, spec in enumerate(bodies):
        spec = dict(spec)
        b["position"][i] = spec.pop("position", (0, 0, 0))
        for key in ("mass", "density", "velocity", "angular_velocity", "orientation", "ccd"):
            if key in spec:
                b[key][i] = spec.pop(key)
        for key, value in spec.items():
            c[key][i] = value
    ids = w.spawn(b, c)
    return w, ids


def state(oracle, body_id):
    s = oracle.states()
    return s[s["body_id"] == body_id][0]


def bullet_scene(ccd):
    return make([dict(shape=R.SHAPE_SPHERE, radius=0.2, mass=0.0),
                 dict(shape=R.SHAPE_SPHERE, radius=0.3, position=(-12.6, 0, 0), velocity=(90, 0, 0), restitution=0.0,
                      ccd=1 if ccd else 0)])


def settle(oracle, steps):
    for _ in range(steps):
        oracle.step(DT)


def test_a_bullet_tunnels_without_ccd_and_stops_at_the_target_with_it():
    w, ids = bullet_scene(False)
    o = O.oracle_from_world(w, DT)
    settle(o, 20)
    assert state(o, ids[1])["position"][0] > 1.0
    w, ids = bullet_scene(True)
    o = O.oracle_from_world(w, DT)
    settle(o, 20)
    x = state(o, ids[1])["position"][0]
    assert -0.6 < x < -0.45, x


def test_a_rod_is_stopped_by_its_leading_face():
    w, ids = make([dict(shape=R.SHAPE_CUBOID, half_extents=(0.05, 5.0, 5.0), mass=0.0),
                   dict(shape=R.SHAPE_CUBOID, half_extents=(1.0, 0.05, 0.05), position=(-4, 0, 0), velocity=(240, 0, 0),
                        restitution=0.0, ccd=1)])
    o = O.oracle_from_world(w, DT)
    o.step(DT)
    assert state(o, ids[1])["position"][0] + 1.0 < 0.05
    settle(o, 20)
    tip = state(o, ids[1])["position"][0] + 1.0
    assert -0.2 < tip < 0.05, tip


def quat_rotate(q, v):
    u, s = np.asarray(q[:3], np.float64), float(q[3])
    v = np.asarray(v, np.float64)
    return 2.0 * np.dot(u, v) * u + (s * s - np.dot(u, u)) * v + 2.0 * s * np.cross(u, v)


def deepest_rod_tip(ccd):
    angle = np.pi / 3.0
    w, ids = make([dict(shape=R.SHAPE_CUBOID, half_extents=(0.05, 2.0, 2.0), mass=0.0, position=(0.9, 0, 0)),
                   dict(shape=R.SHAPE_CUBOID, half_extents=(1.0, 0.05, 0.05),
                        orientation=(0, 0, np.sin(0.5 * angle), np.cos(0.5 * angle)), angular_velocity=(0, 0, -120),
                        ccd=1 if ccd else 0)])
    o = O.oracle_from_world(w, DT)
    deepest = -np.inf
    for _ in range(30):
        o.step(DT)
        s = state(o, ids[1])
        for end in ((1.0, 0, 0), (-1.0, 0, 0)):
            deepest = max(deepest, s["position"][0] + quat_rotate(s["orientation"], end)[0])
    return deepest


def test_continuous_collision_keeps_a_spinning_rod_out_of_the_wall():
    guarded = deepest_rod_tip(True)
    assert 0.85 - 0.1 < guarded < 0.85, guarded
    assert deepest_rod_tip(False) > guarded


def test_a_bullet_stops_at_the_nearest_obstacle_of_a_chain():
    specs = [dict(shape=R.SHAPE_SPHERE, radius=0.15, mass=0.0, position=(-2.0 + i * 0.05, 0, 0)) for i in range(81)]
    specs.append(dict(shape=R.SHAPE_SPHERE, radius=0.3, position=(-12.6, 0, 0), velocity=(90, 0, 0), restitution=0.0,
                      ccd=1))
    w, ids = make(specs)
    o = O.oracle_from_world(w, DT)
    for _ in range(20):
        o.step(DT)
        assert state(o, ids[-1])["position"][0] < -2.0 - 0.4


def test_clearing_the_flag_restores_tunnelling():
    w, ids = bullet_scene(True)
    w.set_ccd(int(ids[1]), False)
    o = O.oracle_from_world(w, DT)
    settle(o, 20)
    assert state(o, ids[1])["position"][0] > 1.0


def test_a_bullet_stops_at_the_anchor_it_may_touch():
    w, ids = make([dict(shape=R.SHAPE_SPHERE, radius=0.5, mass=0.0),
                   dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 8, 0), velocity=(0, -200, 0), ccd=1)])
    o = O.oracle_from_world(w, DT)
    settle(o, 4)
    assert 0.6 < state(o, ids[1])["position"][1] < 1.4


def test_only_a_simulated_body_declares_ccd():
    w, ids = make([dict(shape=R.SHAPE_SPHERE, radius=0.5, mass=0.0), dict(shape=R.SHAPE_SPHERE, radius=0.5)])
    with pytest.raises(DynamisError):
        w.set_ccd(int(ids[0]), True)
    with pytest.raises(DynamisError):
        w.set_ccd(12345, True)
    def flags():
        scene = w.export_scene()
        return int(scene["descs"]["flags"][scene["states"]["body_id"] == ids[1]][0])

    w.set_ccd(int(ids[1]), True)
    assert flags() & R.BODY_CCD
    w.set_ccd(int(ids[1]), False)
    assert not flags() & R.BODY_CCD


def symmetric_targets():
    """A CCD sphere flying between two identical targets placed symmetrically about its path: it
    meets both at the same sweep time, and the library keeps the first pair in collider order."""
    return make([dict(shape=R.SHAPE_SPHERE, radius=0.3, mass=0.0, position=(0, 0, 0.2)),
                 dict(shape=R.SHAPE_SPHERE, radius=0.3, mass=0.0, position=(0, 0, -0.2)),
                 dict(shape=R.SHAPE_SPHERE, radius=0.2, position=(-3, 0, 0), velocity=(120, 0, 0), restitution=0.0,
                      ccd=1)])


def test_symmetric_targets_stop_the_bullet_the_same_way_every_run():
    runs = []
    for _ in range(2):
        w, ids = symmetric_targets()
        o = O.oracle_from_world(w, DT)
        o.step(DT)
        runs.append(state(o, ids[2]))
    assert runs[0]["position"][0] < -0.3  # retreated to the impact, short of the targets
    for field in runs[0].dtype.names:
        assert np.array_equal(runs[0][field], runs[1][field]), field
