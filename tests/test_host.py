"""Host-side scene building through the C ABI (no GPU): hulls, mass properties, records, params.

Restates the behaviours the reference's host tests pin: crates/dynamis-hull/tests/hull.rs:72-215
(box hull, repeated vertices, tetrahedron solid), crates/dynamis-model/tests/mass.rs (closed-form
mass properties), crates/dynamis-abi/tests/records.rs:461-530 (step-parameter mapping).
"""
import numpy as np
import pytest

from dynamis_b200 import DynamisError, World, default_config
from dynamis_b200 import records as R


def cube_corners(h=0.5):
    return np.array([[x, y, z] for x in (-h, h) for y in (-h, h) for z in (-h, h)], np.float32)


def test_config_defaults_follow_physics_config():
    c = default_config()[0]
    assert np.allclose(c["gravity"], [0, -9.81, 0])
    assert (c["substeps"], c["solve_iterations"], c["position_iterations"]) == (2, 8, 10)
    assert np.isclose(c["slop"], 0.005) and np.isclose(c["contact_margin"], 0.02)
    assert np.isclose(c["relaxation"], 0.8) and np.isclose(c["sleep_time"], 0.5)
    assert c["friction_combine"] == 0 and c["restitution_combine"] == 2


def test_box_hull_has_eight_vertices_and_twelve_triangles():
    w = World()
    inner = np.array([[0.1, 0.2, 0.0], [0.0, 0.0, 0.0], [-0.2, 0.1, 0.3]], np.float32)
    src = w.add_hull(np.concatenate([cube_corners(), inner]))
    info = w.hull_info(src)
    assert info["vertices"] == 8
    assert info["triangles"] == 12
    assert np.isclose(info["volume"], 1.0, rtol=1e-5)
    assert np.allclose(info["centroid"], 0.0, atol=1e-6)


def test_hull_handles_repeated_vertices():
    w = World()
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, 0]], np.float32)
    info = w.hull_info(w.add_hull(pts))
    assert info["vertices"] == 4


def test_unit_tetrahedron_solid():
    w = World()
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    info = w.hull_info(w.add_hull(pts))
    assert np.isclose(info["volume"], 1.0 / 6.0, rtol=1e-5)
    assert np.allclose(info["centroid"], 0.25, atol=1e-6)


def test_degenerate_hull_is_refused():
    w = World()
    flat = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0.5, 0.5, 0]], np.float32)
    with pytest.raises(DynamisError) as err:
        w.add_hull(flat)
    assert err.value.status == 6


def spawn_one(shape, density=1000.0, **collider):
    w = World()
    b = R.body_defaults(1)
    b["density"] = density
    c = R.collider_defaults(1)
    c["shape"] = shape
    for k, v in collider.items():
        c[k] = v
    w.spawn(b, c)
    return w.export_scene()


def test_cube_mass_properties():
    s = spawn_one(R.SHAPE_CUBOID, half_extents=(0.5, 0.5, 0.5))
    d = s["descs"][0]
    assert np.isclose(d["inverse_mass"], 1.0 / 1000.0)
    assert np.allclose(d["inertia"], [1000 / 6, 0, 0, 1000 / 6, 0, 1000 / 6], rtol=1e-5)
    assert np.allclose(d["inverse_inertia"], [6 / 1000, 0, 0, 6 / 1000, 0, 6 / 1000], rtol=1e-5)
    assert np.allclose(d["com"], 0.0)


def test_sphere_and_box_mass_properties():
    s = spawn_one(R.SHAPE_SPHERE, radius=0.5)
    mass = 1000.0 * 4.0 / 3.0 * np.pi * 0.125
    d = s["descs"][0]
    assert np.isclose(1.0 / d["inverse_mass"], mass, rtol=1e-5)
    assert np.isclose(d["inertia"][0], 0.4 * mass * 0.25, rtol=1e-5)
    s = spawn_one(R.SHAPE_CUBOID, half_extents=(0.2, 0.5, 0.3))
    d = s["descs"][0]
    m = 1000.0 * 0.4 * 1.0 * 0.6
    assert np.isclose(1.0 / d["inverse_mass"], m, rtol=1e-5)
    assert np.allclose(d["inertia"][[0, 3, 5]], [m * (1.0 + 0.36) / 12, m * (0.16 + 0.36) / 12, m * (0.16 + 1.0) / 12],
                       rtol=1e-5)


def test_hull_of_a_cube_has_the_cube_mass_properties():
    w = World()
    src = w.add_hull(cube_corners())
    b = R.body_defaults(1)
    b["density"] = 1000.0
    c = R.collider_defaults(1)
    c["shape"] = R.SHAPE_HULL
    c["source"] = src
    w.spawn(b, c)
    d = w.export_scene()["descs"][0]
    assert np.isclose(d["inverse_mass"], 1.0 / 1000.0, rtol=1e-5)
    assert np.allclose(d["inertia"][[0, 3, 5]], 1000 / 6, rtol=1e-4)
    assert np.allclose(d["inertia"][[1, 2, 4]], 0.0, atol=1e-3)


def test_static_and_plane_bodies_have_no_mass_and_rows_put_dynamic_bodies_first():
    w = World()
    b = R.body_defaults(3)
    b["mass"] = [0.0, 1.0, 2.0]
    c = R.collider_defaults(3)
    c["shape"] = [R.SHAPE_PLANE, R.SHAPE_SPHERE, R.SHAPE_SPHERE]
    ids = w.spawn(b, c)
    s = w.export_scene()
    assert list(ids) == [0, 1, 2]
    assert s["dynamic"] == 2
    assert list(s["states"]["body_id"]) == [1, 2, 0]
    assert s["descs"]["inverse_mass"][2] == 0.0
    assert list(s["owners"]) == [2, 0, 1]  # collider slots keep spawn order; owners are rows


def test_step_params_mapping():
    w = World(damping=0.1)
    b = R.body_defaults(2)
    c = R.collider_defaults(2)
    w.spawn(b, c)
    p = w.step_params(1.0 / 60.0)[0]
    assert np.isclose(p["dt"], 1 / 60) and np.isclose(p["substep_dt"], np.float32(1 / 60) / np.float32(2))
    assert p["body_count"] == 2 and p["dynamic_count"] == 2 and p["collider_count"] == 2
    assert np.isclose(p["damping"], 0.1) and p["solve_iterations"] == 8 and p["position_iterations"] == 10
    assert np.allclose(p["gravity"], [0, -9.81, 0, 0])


def test_invalid_input_is_refused_not_aborted():
    w = World()
    b = R.body_defaults(1)
    b["collider_count"] = 0
    with pytest.raises(DynamisError):
        w.spawn(b, R.collider_defaults(1))
    with pytest.raises(DynamisError):
        w.step_params(0.0)
    states = np.zeros(2, R.BODY_STATE)
    descs = np.zeros(2, R.BODY_DESCRIPTOR)
    descs["inverse_mass"] = [0.0, 1.0]  # a dynamic row after a static one
    with pytest.raises(DynamisError):
        w.upload_bodies(states, descs, np.zeros(0, R.COLLIDER), np.zeros(0, np.uint32))


def test_contact_frequency_maps_to_relaxation():
    s = spawn_one(R.SHAPE_SPHERE, contact_frequency=10.0)
    assert np.isclose(s["colliders"][0]["relaxation"], 1.0 / (2 * np.pi * 10.0))
    s = spawn_one(R.SHAPE_SPHERE)
    assert s["colliders"][0]["relaxation"] == 0.0
