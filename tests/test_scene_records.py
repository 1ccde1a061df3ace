"""The records a world uploads, built two ways: by the library (dyn_spawn_bodies, dyn_add_hull,
dyn_export_scene, dyn_step_params_for) and by the oracle's own restatement of the reference's spawn
path (oracle/scene.cpp: dynamis-hull's hull() and solid(), compute_mass_properties,
BodyStateRecord::initial, BodyDescriptorRecord::build, ColliderRecord::build, the shape roles'
scale rules, StepParamsRecord::new, the row census). They must agree byte for byte: body states,
descriptors (mass, centre of mass, inertia and its inverse), colliders, owners, hull sources,
hull vertices and step parameters.

The stress scene mixes every convex shape in compound bodies with offset and rotated colliders,
uniform and non-uniform scales, sensors, density and fixed-mass bodies, static and kinematic ones.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from dynamis_b200 import records as R
from oracle import oracle as O

DT = 1.0 / 60.0


def stress_scene(seed=7, n=40):
    rng = np.random.default_rng(seed)
    bodies = R.body_defaults(n)
    parts, first = [], 0
    hulls = [rng.normal(size=(20, 3)).astype(np.float32), rng.normal(size=(12, 3)).astype(np.float32)]
    shapes = [R.SHAPE_SPHERE, R.SHAPE_CUBOID, R.SHAPE_CAPSULE, R.SHAPE_CYLINDER, R.SHAPE_HULL]
    for b in range(n):
        k = int(rng.integers(1, 4))
        c = R.collider_defaults(k)
        for j in range(k):
            c["shape"][j] = shapes[int(rng.integers(0, len(shapes)))]
            c["radius"][j] = rng.uniform(0.1, 0.6)
            c["half_height"][j] = rng.uniform(0.1, 0.5)
            c["half_extents"][j] = rng.uniform(0.1, 0.6, 3)
            c["source"][j] = int(rng.integers(0, 2))
            c["offset"][j] = rng.uniform(-0.5, 0.5, 3)
            q = rng.normal(size=4)
            c["rotation"][j] = q / np.linalg.norm(q)
            c["scale"][j] = rng.uniform(0.5, 1.5, 3) if rng.random() < 0.5 else rng.uniform(0.5, 1.5)
            c["sensor"][j] = 1 if rng.random() < 0.1 else 0
            c["friction"][j] = rng.uniform(0.1, 0.9)
        parts.append(c)
        bodies["collider_first"][b] = first
        bodies["collider_count"][b] = k
        first += k
        bodies["position"][b] = rng.uniform(-5, 5, 3)
        q = rng.normal(size=4)
        bodies["orientation"][b] = q / np.linalg.norm(q)
        mode = rng.random()
        if mode < 0.4:
            bodies["density"][b] = rng.uniform(200, 2000)
        elif mode < 0.8:
            bodies["mass"][b] = rng.uniform(0.5, 5)
        elif mode < 0.9:
            bodies["mass"][b] = 0.0
        else:
            bodies["kinematic"][b] = 1
    return scenes.Scene(bodies, np.concatenate(parts), hulls, "stress")


SCENES = {
    "stress": lambda: stress_scene(),
    "falling_boxes": lambda: scenes.falling_boxes(seed=0),
    "mixed_pile_216": lambda: scenes.mixed_pile(side=6, seed=1),
    "random_mix_24": lambda: scenes.random_mix(24, seed=5),
    "batched_worlds_8": lambda: scenes.batched_worlds(8),
    "tower": lambda: scenes.tower_world(seed=3),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_the_library_uploads_the_records_the_reference_would(name):
    scene = SCENES[name]()
    world = World()
    scene.build(world)
    mine = world.export_scene()
    params = world.step_params(DT)
    world.close()
    theirs = O.scene_records(scene.bodies, scene.colliders, scene.hulls, scene.worlds, dt=DT)
    for key in ("states", "descs", "colliders", "owners", "sources", "vertices"):
        assert mine[key].tobytes() == theirs[key].tobytes(), f"{name}: {key} differ"
    assert mine["dynamic"] == theirs["dynamic"]
    assert params.tobytes() == theirs["params"].tobytes(), f"{name}: step parameters differ"
    if "body_world" in mine:
        assert np.array_equal(mine["body_world"], theirs["body_world"])
