"""Batched worlds on the CPU: sub-worlds of one batch step exactly as the same worlds alone.

A batch puts every body in a sub-world; the sub-world is mixed into the grid keys and bodies of
different sub-worlds never pair. Since the candidate pairs are exactly the overlapping swept boxes,
whatever the grid, each sub-world of a batch must step bit for bit as the same world stepped alone.
"""
import numpy as np
import pytest

from dynamis_b200 import DynamisError, World, scenes
from oracle.oracle import OracleWorld, oracle_from_world

DT = 1.0 / 60.0


def parts():
    return [scenes.random_mix(12, seed=21), scenes.box_lattice(27, seed=5), scenes.hanging_chains(1, 2, 4),
            scenes.random_mix(9, seed=22)]


def step_oracle(scene_obj, steps, dt=DT):
    w = World()
    scene_obj.build(w)
    o = oracle_from_world(w, dt)
    for _ in range(steps):
        o.step(dt)
    states = o.states()
    o.close()
    w.close()
    return states


def test_each_sub_world_steps_as_it_would_alone():
    ps = parts()
    alone = [step_oracle(p, 20) for p in ps]
    together = step_oracle(scenes.batch(ps), 20)
    by_id = {int(s["body_id"]): s for s in together}
    base = 0
    for p, states in zip(ps, alone):
        for s in states:
            t = by_id[int(s["body_id"]) + base]
            for f in ("position", "orientation", "velocity", "angular_velocity"):
                assert np.array_equal(s[f], t[f]), f
        base += len(p.bodies)


def test_one_sub_world_keeps_the_single_world_keys():
    sc = scenes.random_mix(16, seed=8)
    a = World()
    sc.build(a)
    b = World()
    solo = scenes.batch([sc])
    solo.build(b)
    oa, ob = oracle_from_world(a, DT), oracle_from_world(b, DT)
    oa.step(DT)
    ob.step(DT)
    assert np.array_equal(oa.entries()[0], ob.entries()[0])
    a.close()
    b.close()


def test_joints_across_sub_worlds_are_refused():
    sc = scenes.batch([scenes.sphere_row(2), scenes.sphere_row(2)])
    w = World()
    ids = sc.build(w)
    w.add_ball_joint(int(ids[0]), int(ids[2]), (0, 0, 0), (0, 0, 0))
    with pytest.raises(DynamisError):
        w.export_scene()
    w.close()
