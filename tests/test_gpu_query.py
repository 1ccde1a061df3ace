"""Scene queries on the GPU (dyn_query; query.cuh) against the oracle.

The oracle rebuilds the grid index from the same states and restates the candidate walk over it
(binary searches in the sorted keys where the library uses its cell table), so agreement checks the
walk, the tests and the selection together. Compared
per query: hit_base, count, overflow; per hit: body id and generation, the candidate (collider),
the triangle, and distance / point / normal within 1e-5 relative + 1e-6 absolute.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from dynamis_b200 import records as R
from oracle import oracle as O
from test_query import make, static_sphere

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-5, 1e-6


def close(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= ATOL + RTOL * np.abs(b))


def oracle_now(world, dt=1.0 / 60.0):
    """The oracle over the device's current states."""
    scene = world.export_scene()
    scene["states"] = world.read_states()
    return O.OracleWorld(scene, world.step_params(dt))


def compare(world, queries, oracle=None):
    batch = np.concatenate(queries)
    gq, gh = world.query(batch)
    oq, oh = (oracle or oracle_now(world)).query(batch)
    for name in ("hit_base", "count", "overflow"):
        assert np.array_equal(gq[name], oq[name]), f"query {name} differs: {gq[name]} vs {oq[name]}"
    for i, r in enumerate(oq):
        g = gh[r["hit_base"]: r["hit_base"] + r["count"]]
        o = oh[r["hit_base"]: r["hit_base"] + r["count"]]
        for name in ("body_id", "body_generation", "scene_target", "triangle", "surface"):
            assert np.array_equal(g[name], o[name]), f"query {i} (kind {r['kind']}): hit {name} differs"
        for name in ("distance", "point", "normal"):
            assert close(g[name], o[name]), f"query {i} (kind {r['kind']}): hit {name} differs"
    return gq, gh


def test_the_reference_query_scenes_match_the_oracle():
    w, _ = make([static_sphere(0.5, (0, 0, 2)), static_sphere(0.5, (0, 0, 10)), static_sphere(1.0, (5, 0, 0)),
                 dict(shape=R.SHAPE_CUBOID, half_extents=(1, 1, 1), mass=0.0, position=(-5, 0, 0)),
                 dict(shape=R.SHAPE_CYLINDER, radius=1.0, half_height=1.0, mass=0.0, position=(0, 0, -6)),
                 dict(shape=R.SHAPE_CAPSULE, radius=0.5, half_height=1.0, scale=(2, 1, 1), mass=0.0, position=(10, 0, 0))])
    sphere = dict(kind=R.SHAPE_SPHERE, radius=0.3)
    compare(w, [R.ray_query((0, 0, 0), (0, 0, 1), 20.0), R.ray_query((0, 0, 0), (0, 0, 1), 5.0),
                R.ray_query((0, 0, 2), (0, 0, 1), 20.0), R.sphere_query((0, 0, 2.8), 0.5),
                R.cuboid_query((-4.1, 0.99, 0.9), (0.2, 0.2, 0.2)), R.point_query((5.5, 0, 0)),
                R.sweep_query(sphere, (0, 0, 0, 1), (0, 0, 4), (0, 0, 1), 30.0),
                R.ray_query((0.5, 5, -6), (0, -1, 0), 20.0), R.ray_query((10.6, 5, 0), (0, -1, 0), 20.0),
                R.ray_query((-20, 0, 0), (1, 0, 0), 60.0, R.query_filter(max_hits=8))])
    w.close()


def random_queries(rng, count, extent, hull_source):
    shapes = [dict(kind=R.SHAPE_SPHERE, radius=0.3), dict(kind=R.SHAPE_CUBOID, half_extents=(0.3, 0.2, 0.4)),
              dict(kind=R.SHAPE_CAPSULE, radius=0.2, half_height=0.3), dict(kind=R.SHAPE_CYLINDER, radius=0.3, half_height=0.2),
              dict(kind=R.SHAPE_HULL, source=hull_source)]
    out = []
    for i in range(count):
        origin = rng.uniform(-extent, extent, 3) + (0, extent, 0)
        direction = rng.normal(size=3)
        quat = rng.normal(size=4)
        quat /= np.linalg.norm(quat)
        filt = R.query_filter(max_hits=int(rng.integers(1, 9)))
        kind = i % 6
        if kind == 0:
            out.append(R.ray_query(origin, direction, float(rng.uniform(1, 3 * extent)), filt))
        elif kind == 1:
            out.append(R.sphere_query(origin, float(rng.uniform(0.2, 1.5)), filt))
        elif kind == 2:
            out.append(R.point_query(origin, filt))
        elif kind == 3:
            out.append(R.cuboid_query(origin, rng.uniform(0.2, 1.0, 3), filt))
        elif kind == 4:
            out.append(R.overlap_query(shapes[int(rng.integers(0, 5))], quat, origin, filt))
        else:
            out.append(R.sweep_query(shapes[int(rng.integers(0, 5))], quat, origin, direction,
                                     float(rng.uniform(0.5, 2 * extent)), filt))
    return out


@pytest.mark.parametrize("seed", [3, 8])
def test_random_queries_on_a_stepped_heap_match_the_oracle(seed):
    w = World()
    scenes.random_mix(60, seed=seed).build(w)
    for _ in range(10):
        w.step(1.0 / 60.0)
    w.wait()
    rng = np.random.default_rng(seed)
    gq, gh = compare(w, random_queries(rng, 240, 3.0, 0))
    assert gq["count"].sum() > 100  # the batch does hit things
    w.close()


def test_queries_on_a_formed_pile():
    # 4,096 mixed bodies after 90 steps: the grid walk over a dense scene, its levels and cells
    w = World()
    scenes.mixed_pile(16, seed=1).build(w)
    for _ in range(90):
        w.step(1.0 / 60.0)
    w.wait()
    rng = np.random.default_rng(5)
    gq, _ = compare(w, random_queries(rng, 96, 10.0, 0))
    assert gq["count"].sum() > 50
    w.close()
