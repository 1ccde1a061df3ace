"""Scene queries on the oracle: the reference's query behaviours, restated
(crates/dynamis-world/tests/suite/query.rs).

  * a ray hits the nearest body and faces the ray; misses out of range and behind   :15-69
  * a ray from inside a body returns its exit distance                              :70-89
  * a sphere query reports penetration (-0.2) and misses                            :90-107
  * a cuboid query reports overlap and misses outside                               :108-119
  * a convex overlap separates along the face the narrowphase solves                :120-141
  * a sweep stops at the surface (7.7) facing the swept shape                       :152-178
  * cylinder cap and side rays, capsule cross sections, scaled primitives           :352-459
  * multi-hit queries in distance order, truncation and the overflow flag           :678-712, 1144-1257
  * point queries inside, outside and on the surface                                :943-966
  * the body filters (static, sensors, include, exclude, group and mask)            :533-677, 997-1020
The GPU path is compared with the oracle in test_gpu_query.py.
"""
import numpy as np
import pytest

from dynamis_b200 import World
from dynamis_b200 import records as R
from oracle import oracle as O

STATIC = {"gravity": (0.0, 0.0, 0.0), "damping": 0.0, "angular_damping": 0.0}


def make(bodies, config=None):
    w = World(**(config or STATIC))
    n = len(bodies)
    b = R.body_defaults(n)
    c = R.collider_defaults(n)
    for i, spec in enumerate(bodies):
        spec = dict(spec)
        b["position"][i] = spec.pop("position", (0, 0, 0))
        for key in ("mass", "density", "velocity", "angular_velocity", "orientation", "kinematic"):
            if key in spec:
                b[key][i] = spec.pop(key)
        for key, value in spec.items():
            c[key][i] = value
    ids = w.spawn(b, c)
    return w, ids


def static_sphere(radius, position, **extra):
    return dict(shape=R.SHAPE_SPHERE, radius=radius, mass=0.0, position=position, **extra)


def run(world, queries):
    o = O.oracle_from_world(world, 1.0 / 60.0)
    q, hits = o.query(np.concatenate(queries))
    return [hits[r["hit_base"]: r["hit_base"] + r["count"]] for r in q], q


def test_a_ray_hits_the_nearest_body_and_faces_the_ray():
    w, ids = make([static_sphere(0.5, (0, 0, 2)), static_sphere(0.5, (0, 0, 10))])
    (hits,), _ = run(w, [R.ray_query((0, 0, 0), (0, 0, 1), 20.0, R.query_filter(max_hits=1))])
    assert hits[0]["body_id"] == ids[0]
    assert abs(hits[0]["distance"] - 1.5) < 1e-3 and abs(hits[0]["point"][2] - 1.5) < 1e-3
    assert abs(hits[0]["normal"][2] + 1.0) < 1e-3


def test_rays_miss_out_of_range_and_behind():
    w, _ = make([static_sphere(0.5, (0, 0, 10))])
    (short,), _ = run(w, [R.ray_query((0, 0, 0), (0, 0, 1), 5.0)])
    assert len(short) == 0
    w, _ = make([static_sphere(0.5, (0, 0, -5))])
    (behind,), _ = run(w, [R.ray_query((0, 0, 0), (0, 0, 1), 20.0)])
    assert len(behind) == 0


def test_a_ray_from_inside_returns_the_exit_distance():
    w, ids = make([static_sphere(0.5, (0, 0, 0))])
    (hits,), _ = run(w, [R.ray_query((0, 0, 0), (0, 0, 1), 20.0)])
    assert hits[0]["body_id"] == ids[0] and abs(hits[0]["distance"] - 0.5) < 1e-3


def test_a_sphere_query_reports_penetration_and_misses():
    w, ids = make([static_sphere(0.5, (0, 0, 0))])
    (overlap, miss), _ = run(w, [R.sphere_query((0, 0, 0.8), 0.5), R.sphere_query((0, 0, 5), 0.5)])
    assert overlap[0]["body_id"] == ids[0] and abs(overlap[0]["distance"] + 0.2) < 1e-3
    assert len(miss) == 0


def test_a_cuboid_query_reports_overlap_and_misses_outside():
    w, _ = make([static_sphere(1.0, (0, 0, 0))])
    (inside, outside), _ = run(w, [R.cuboid_query((0, 0, 0), (2, 2, 2)), R.cuboid_query((0, 0, 10), (1, 1, 1))])
    assert len(inside) == 1 and len(outside) == 0


def test_a_convex_overlap_separates_along_the_face():
    w, ids = make([dict(shape=R.SHAPE_CUBOID, half_extents=(1, 1, 1), mass=0.0)])
    (hits,), _ = run(w, [R.cuboid_query((0.9, 0.99, 0.9), (0.2, 0.2, 0.2))])
    assert hits[0]["body_id"] == ids[0]
    assert abs(hits[0]["normal"][1] - 1.0) < 1e-3 and hits[0]["distance"] < 0.0


def test_a_sweep_stops_at_the_surface():
    w, ids = make([static_sphere(2.0, (0, 0, 10))])
    sphere = dict(kind=R.SHAPE_SPHERE, radius=0.3)
    (hits,), _ = run(w, [R.sweep_query(sphere, (0, 0, 0, 1), (0, 0, 0), (0, 0, 1), 30.0)])
    assert hits[0]["body_id"] == ids[0]
    assert abs(hits[0]["distance"] - 7.7) < 0.05 and abs(hits[0]["normal"][2] + 1.0) < 1e-3


def test_cylinder_cap_and_side_rays():
    w, _ = make([dict(shape=R.SHAPE_CYLINDER, radius=1.0, half_height=1.0, mass=0.0)])
    caps = [R.ray_query((x, 5, 0), (0, -1, 0), 20.0) for x in (0.0, 0.5, 0.9, 0.99)]
    sides = [R.ray_query((-5, h, 0), (1, 0, 0), 20.0) for h in (-1.0, -0.5, 0.0, 0.5, 0.99)]
    found, _ = run(w, caps + sides)
    for hits, x in zip(found[:4], (0.0, 0.5, 0.9, 0.99)):
        assert abs(hits[0]["distance"] - 4.0) < 1e-3 and abs(hits[0]["point"][1] - 1.0) < 1e-3
        assert abs(hits[0]["point"][0] - x) < 1e-3 and abs(hits[0]["normal"][1] - 1.0) < 1e-3
    for hits in found[4:]:
        assert abs(hits[0]["distance"] - 4.0) < 1e-3 and abs(hits[0]["point"][0] + 1.0) < 1e-3
        assert abs(hits[0]["normal"][0] + 1.0) < 1e-3


def test_a_capsule_ray_reaches_every_cross_section():
    w, _ = make([dict(shape=R.SHAPE_CAPSULE, radius=0.08, half_height=2.0, mass=0.0)])
    heights = (-2.0, -1.875, -0.75, -0.25, 0.125, 0.375, 1.0, 1.875)
    found, _ = run(w, [R.ray_query((-5, h, 0), (1, 0, 0), 20.0) for h in heights])
    for hits in found:
        assert abs(hits[0]["distance"] - 4.92) < 1e-3 and abs(hits[0]["point"][0] + 0.08) < 1e-3
        assert abs(hits[0]["normal"][0] + 1.0) < 1e-3


def test_a_scaled_primitive_ray_lands_on_its_scaled_surface():
    w, _ = make([dict(shape=R.SHAPE_SPHERE, radius=0.5, scale=(2, 1, 1), mass=0.0),
                 dict(shape=R.SHAPE_CAPSULE, radius=0.5, half_height=1.0, scale=(2, 1, 1), mass=0.0, position=(10, 0, 0))])
    (sphere, capsule), _ = run(w, [R.ray_query((0.6, 5, 0), (0, -1, 0), 20.0), R.ray_query((10.6, 5, 0), (0, -1, 0), 20.0)])
    assert abs(sphere[0]["distance"] - 4.6) < 1e-3 and abs(sphere[0]["point"][1] - 0.4) < 1e-3
    assert abs(capsule[0]["distance"] - 3.6) < 1e-3 and abs(capsule[0]["point"][1] - 1.4) < 1e-3


def test_multi_hit_queries_report_in_distance_order_and_flag_truncation():
    w, ids = make([static_sphere(0.4, (0, 0, 2.0)), static_sphere(0.4, (0, 0, 2.7)), static_sphere(0.4, (0, 0, 3.4))])
    found, q = run(w, [R.sphere_query((0, 0, 2.7), 1.2, R.query_filter(max_hits=4)),
                       R.sphere_query((0, 0, 2.7), 1.2, R.query_filter(max_hits=1)),
                       R.ray_query((0, 0, 0), (0, 0, 1), 20.0, R.query_filter(max_hits=3)),
                       R.ray_query((0, 0, 0), (0, 0, 1), 20.0, R.query_filter(max_hits=2))])
    assert len(found[0]) == 3 and np.all(np.diff(found[0]["distance"]) >= 0) and q["overflow"][0] == 0
    assert len(found[1]) == 1 and q["overflow"][1] == 1
    assert list(found[2]["body_id"]) == list(ids) and q["overflow"][2] == 0
    assert list(found[3]["body_id"]) == list(ids[:2]) and q["overflow"][3] == 1
    assert list(q["hit_base"]) == [0, 4, 5, 8]


def test_point_queries_inside_outside_and_on_the_surface():
    w, ids = make([static_sphere(0.5, (0, 0, 0))])
    (inside, outside, edge), _ = run(w, [R.point_query((0.1, 0, 0)), R.point_query((5, 0, 0)), R.point_query((0.5, 0, 0))])
    assert inside[0]["body_id"] == ids[0] and len(outside) == 0 and len(edge) == 1


def test_filters_select_bodies():
    w, ids = make([static_sphere(0.5, (0, 0, 2)),
                   dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 0, 4)),  # dynamic
                   static_sphere(0.5, (0, 0, 6), sensor=1),
                   dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 0, 8), collision_group=4, collision_mask=4)])
    ray = lambda **f: R.ray_query((0, 0, 0), (0, 0, 1), 20.0, R.query_filter(max_hits=8, **f))
    found, _ = run(w, [ray(), ray(ignore_static=True), ray(ignore_sensors=False),
                       ray(include=(int(ids[1]), 0)), ray(exclude=(int(ids[0]), 0)), ray(group=4, mask=4)])
    assert list(found[0]["body_id"]) == [ids[0], ids[1], ids[3]]  # sensors ignored by default
    assert list(found[1]["body_id"]) == [ids[1], ids[3]]
    assert list(found[2]["body_id"]) == [ids[0], ids[1], ids[2], ids[3]]
    assert list(found[3]["body_id"]) == [ids[1]]
    assert list(found[4]["body_id"]) == [ids[1], ids[3]]
    assert list(found[5]["body_id"]) == [ids[3]]


def test_the_host_accepts_every_record_the_builders_make():
    # validation runs on the host before any device work: a valid batch gets past it (and on a
    # machine without a GPU stops at the device), an invalid one is refused as invalid
    from dynamis_b200._native import DynamisError
    w, _ = make([static_sphere(0.5, (0, 0, 0))])
    probe = dict(kind=R.SHAPE_CAPSULE, radius=0.2, half_height=0.3)
    valid = np.concatenate([R.ray_query((0, 0, 0), (0, 0, 1), 20.0), R.sphere_query((0, 0, 0), 0.5),
                            R.point_query((0, 0, 0)), R.cuboid_query((0, 0, 0), (1, 1, 1)),
                            R.overlap_query(probe, (0, 0, 0, 1), (0, 0, 0)),
                            R.sweep_query(probe, (0, 0, 0, 1), (0, 0, 0), (1, 0, 0), 2.0)])
    try:
        w.query(valid)
    except DynamisError as e:
        assert e.status != 1, "a valid query batch was refused as invalid"
    for bad in (R.ray_query((0, 0, 0), (0, 0, 1), -1.0), R.sphere_query((0, 0, 0), 0.0),
                R.overlap_query(probe, (0, 0, 0, 2), (0, 0, 0)), R.overlap_query(dict(kind=R.SHAPE_PLANE), (0, 0, 0, 1), (0, 0, 0))):
        with pytest.raises(DynamisError) as e:
            w.query(bad)
        assert e.value.status == 1


def test_invalid_queries_are_refused():
    from dynamis_b200._native import DynamisError
    w, _ = make([static_sphere(0.5, (0, 0, 0))])
    bad = R.ray_query((0, 0, 0), (0, 0, 0), 20.0)
    with pytest.raises(DynamisError):
        w.query(bad)  # refused on the host, before any device work
