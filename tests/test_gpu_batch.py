"""Batched worlds on the GPU: one dyn_step advances every sub-world, each exactly as alone.

The batch is checked against the oracle every step (all products), and against the same worlds
stepped one by one on the GPU (body states bit for bit).
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from test_batch import parts
from test_gpu_parity import compare_step
from oracle.oracle import oracle_from_world

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def test_a_batch_matches_the_oracle_every_step():
    w = World()
    scenes.batch(parts()).build(w)
    o = oracle_from_world(w, DT)
    for step in range(40):
        w.step(DT)
        o.step(DT)
        w.wait()
        compare_step(w, o, step)
    o.close()
    w.close()


def test_a_batch_steps_each_world_as_the_world_alone():
    ps = parts()
    batch = World()
    scenes.batch(ps).build(batch)
    alone = []
    for p in ps:
        w = World()
        p.build(w)
        alone.append(w)
    for _ in range(40):
        batch.step(DT)
        for w in alone:
            w.step(DT)
    batch.wait()
    together = {int(s["body_id"]): s for s in batch.read_states()}
    base = 0
    for p, w in zip(ps, alone):
        w.wait()
        for s in w.read_states():
            t = together[int(s["body_id"]) + base]
            for f in ("position", "orientation", "velocity", "angular_velocity", "sleeping"):
                assert np.array_equal(s[f], t[f]), f
        base += len(p.bodies)
        w.close()
    batch.close()
