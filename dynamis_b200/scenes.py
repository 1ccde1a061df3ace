"""Seeded synthetic scenes: the benchmark workloads and the small scenes the tests pin.

The workloads are the benchmark scenes of this path (lattices of boxes, spheres and hulls falling
onto a ground plane, hanging chains, batches of small worlds); no dataset is involved. Every random draw comes from
numpy.random.default_rng(seed), so a seed fixes a scene bit for bit.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import records as R


# a ball joint between two bodies of a scene (indices into Scene.bodies), anchors in body frames
JOINT = np.dtype([("first", "<u4"), ("second", "<u4"), ("anchor_a", "<f4", 3), ("anchor_b", "<f4", 3)])


@dataclass
class Scene:
    bodies: np.ndarray                      # BODY_DESC
    colliders: np.ndarray                   # COLLIDER_DESC; hull colliders index `hulls`
    hulls: list = field(default_factory=list)  # float32 (m, 3) point sets
    name: str = "scene"
    joints: np.ndarray | None = None        # JOINT rows: ball joints added after the bodies
    worlds: np.ndarray | None = None        # sub-world of every body (a batch of independent worlds)

    @property
    def body_count(self) -> int:
        return len(self.bodies)

    def build(self, world) -> np.ndarray:
        """Adds the hull sources and spawns every body into `world`; returns the body ids."""
        colliders = self.colliders.copy()
        if self.hulls:
            sources = np.array([world.add_hull(points) for points in self.hulls], np.uint32)
            is_hull = colliders["shape"] == R.SHAPE_HULL
            colliders["source"][is_hull] = sources[colliders["source"][is_hull]]
        ids = world.spawn(self.bodies, colliders)
        if self.worlds is not None:
            by_id = np.zeros(int(ids.max()) + 1, np.uint32)
            by_id[ids] = self.worlds
            world.set_body_worlds(by_id)
        if self.joints is not None and len(self.joints):
            world.add_constraints(ball_joint_records(ids[self.joints["first"]], ids[self.joints["second"]],
                                                     self.joints["anchor_a"], self.joints["anchor_b"]))
        return ids


def ball_joint_records(first_ids, second_ids, anchor_a, anchor_b) -> np.ndarray:
    """ConstraintDescriptorRecords of ConstraintDesc::ball joints with the reference's defaults
    (collisions disabled between the pair, warm start, axis +y), as dyn_add_ball_joint builds them."""
    rec = np.zeros(len(first_ids), R.CONSTRAINT_DESCRIPTOR)
    rec["kind"] = R.CONSTRAINT_BALL
    rec["first_body_id"] = first_ids
    rec["second_body_id"] = second_ids
    rec["flags"] = R.CONSTRAINT_DISABLE_COLLISIONS | R.CONSTRAINT_WARM_START
    rec["anchor_a"] = anchor_a
    rec["anchor_b"] = anchor_b
    rec["axis_a"] = (0.0, 1.0, 0.0)
    rec["swing_a"] = np.float32(np.pi)
    rec["swing_b"] = np.float32(np.pi)
    rec["gear_ratio"] = 1.0
    return rec


def yaw_quaternions(angles: np.ndarray) -> np.ndarray:
    q = np.zeros((len(angles), 4), np.float64)
    q[:, 1] = np.sin(angles / 2)
    q[:, 3] = np.cos(angles / 2)
    return q.astype(np.float32)


def uniform_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniformly distributed rotations (Shoemake, "Uniform random rotations", Graphics Gems III)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
    q = np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2), b * np.sin(2 * np.pi * u3),
                  b * np.cos(2 * np.pi * u3)], axis=1)
    return q.astype(np.float32)


def _ground(bodies: np.ndarray, colliders: np.ndarray, height: float = 0.0, friction: float = 0.5,
            restitution: float = 0.0):
    """Appends a static body carrying a ground plane (normal +y) at the given height."""
    b = R.body_defaults(1)
    b["position"][0] = (0.0, height, 0.0)
    b["mass"] = 0.0
    b["collider_first"] = len(colliders)
    c = R.collider_defaults(1)
    c["shape"] = R.SHAPE_PLANE
    c["friction"] = friction
    c["restitution"] = restitution
    return np.concatenate([bodies, b]), np.concatenate([colliders, c])


def falling_boxes(seed: int = 0, side: int = 10, spacing: float = 1.1) -> Scene:
    """1,000 unit cubes (half-extent 0.5 m, density 1000) on a 10x10x10 lattice at 1.1 m spacing,
    +-0.05 m position jitter and a random yaw each, at rest above a static ground plane at y = 0;
    friction 0.5, restitution 0."""
    rng = np.random.default_rng(seed)
    n = side ** 3
    i, j, k = np.meshgrid(np.arange(side), np.arange(side), np.arange(side), indexing="ij")
    base = np.stack([(i.ravel() - (side - 1) / 2) * spacing, 0.6 + j.ravel() * spacing,
                     (k.ravel() - (side - 1) / 2) * spacing], axis=1)
    pos = base + rng.uniform(-0.05, 0.05, size=(n, 3))
    bodies = R.body_defaults(n)
    bodies["position"] = pos.astype(np.float32)
    bodies["orientation"] = yaw_quaternions(rng.uniform(0.0, 2 * np.pi, n))
    bodies["density"] = 1000.0
    colliders = R.collider_defaults(n)
    colliders["shape"] = R.SHAPE_CUBOID
    colliders["half_extents"] = 0.5
    colliders["friction"] = 0.5
    colliders["restitution"] = 0.0
    bodies, colliders = _ground(bodies, colliders, 0.0, 0.5, 0.0)
    return Scene(bodies, colliders, [], f"falling_boxes_{n}")


def resting_field(side: int = 512, spacing: float = 1.1) -> Scene:
    """side x side unit cubes (half-extent 0.5 m, density 1000) standing on a static ground plane at
    1.1 m spacing, none touching another: every box falls asleep within a second and the world then
    rests (the kept grid runs' case)."""
    n = side * side
    i, k = np.meshgrid(np.arange(side), np.arange(side), indexing="ij")
    pos = np.stack([(i.ravel() - (side - 1) / 2) * spacing, np.full(n, 0.5), (k.ravel() - (side - 1) / 2) * spacing],
                   axis=1)
    bodies = R.body_defaults(n)
    bodies["position"] = pos.astype(np.float32)
    bodies["density"] = 1000.0
    colliders = R.collider_defaults(n)
    colliders["shape"] = R.SHAPE_CUBOID
    colliders["half_extents"] = 0.5
    bodies, colliders = _ground(bodies, colliders, 0.0, 0.5, 0.0)
    return Scene(bodies, colliders, [], f"resting_field_{n}")


def mixed_pile(side: int = 64, seed: int = 1, spacing: float = 1.3) -> Scene:
    """side^3 bodies on a lattice at 1.3 m spacing with +-0.1 m jitter and uniform random
    orientations: 50% boxes (half-extents U[0.2, 0.6] per axis), 30% spheres (radius U[0.2, 0.5]),
    20% convex hulls (16-32 points uniform on the unit sphere, scaled U[0.3, 0.6]); density 1000,
    friction 0.5, restitution 0.1, over a ground plane at y = 0. side = 64 gives 262,144 bodies."""
    rng = np.random.default_rng(seed)
    n = side ** 3
    i, j, k = np.meshgrid(np.arange(side), np.arange(side), np.arange(side), indexing="ij")
    base = np.stack([(i.ravel() - (side - 1) / 2) * spacing, 1.2 + j.ravel() * spacing,
                     (k.ravel() - (side - 1) / 2) * spacing], axis=1)
    pos = base + rng.uniform(-0.1, 0.1, size=(n, 3))
    kind = rng.random(n)
    shape = np.where(kind < 0.5, R.SHAPE_CUBOID, np.where(kind < 0.8, R.SHAPE_SPHERE, R.SHAPE_HULL)).astype(np.uint32)
    bodies = R.body_defaults(n)
    bodies["position"] = pos.astype(np.float32)
    bodies["orientation"] = uniform_quaternions(rng, n)
    bodies["density"] = 1000.0
    colliders = R.collider_defaults(n)
    colliders["shape"] = shape
    colliders["friction"] = 0.5
    colliders["restitution"] = 0.1
    boxes = shape == R.SHAPE_CUBOID
    colliders["half_extents"][boxes] = rng.uniform(0.2, 0.6, size=(int(boxes.sum()), 3)).astype(np.float32)
    spheres = shape == R.SHAPE_SPHERE
    colliders["radius"][spheres] = rng.uniform(0.2, 0.5, size=int(spheres.sum())).astype(np.float32)
    hull_rows = np.nonzero(shape == R.SHAPE_HULL)[0]
    hulls = []
    for index, row in enumerate(hull_rows):
        m = int(rng.integers(16, 33))
        d = rng.normal(size=(m, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        scale = rng.uniform(0.3, 0.6)
        hulls.append((d * scale).astype(np.float32))
        colliders["source"][row] = index
        colliders["radius"][row] = 0.0
    bodies, colliders = _ground(bodies, colliders, 0.0, 0.5, 0.1)
    return Scene(bodies, colliders, hulls, f"mixed_pile_{n}")


def sphere_row(count: int, radius: float = 0.5, gap: float = -0.05, height: float = 5.0, gravity: bool = False) -> Scene:
    """`count` spheres in a row along x, neighbours overlapping by -gap (a 16-sphere chain has 15 pairs)."""
    bodies = R.body_defaults(count)
    bodies["position"][:, 0] = np.arange(count) * (2 * radius + gap)
    bodies["position"][:, 1] = height
    if not gravity:
        bodies["gravity_scale"] = 0.0
    colliders = R.collider_defaults(count)
    colliders["radius"] = radius
    return Scene(bodies, colliders, [], f"sphere_row_{count}")


def crowd(count: int, seed: int = 3) -> Scene:
    """`count` unit boxes resting on a wide floor box, none touching each other."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(np.sqrt(count)))
    bodies = R.body_defaults(count)
    idx = np.arange(count)
    bodies["position"][:, 0] = (idx % side) * 3.0
    bodies["position"][:, 2] = (idx // side) * 3.0
    bodies["position"][:, 1] = 0.5
    bodies["orientation"] = yaw_quaternions(rng.uniform(0, 2 * np.pi, count))
    colliders = R.collider_defaults(count)
    colliders["shape"] = R.SHAPE_CUBOID
    colliders["half_extents"] = 0.5
    floor = R.body_defaults(1)
    floor["mass"] = 0.0
    floor["position"][0] = (side * 1.5, -0.5, side * 1.5)
    floor["collider_first"] = count
    fc = R.collider_defaults(1)
    fc["shape"] = R.SHAPE_CUBOID
    fc["half_extents"] = (side * 2.0, 0.5, side * 2.0)
    return Scene(np.concatenate([bodies, floor]), np.concatenate([colliders, fc]), [], f"crowd_{count}")


def box_tower(levels: int = 8, half: float = 0.5, gap: float = 0.0) -> Scene:
    """A single column of unit boxes resting on a ground plane."""
    bodies = R.body_defaults(levels)
    bodies["position"][:, 1] = half + np.arange(levels) * (2 * half + gap)
    bodies["density"] = 1000.0
    colliders = R.collider_defaults(levels)
    colliders["shape"] = R.SHAPE_CUBOID
    colliders["half_extents"] = half
    bodies, colliders = _ground(bodies, colliders)
    return Scene(bodies, colliders, [], f"box_tower_{levels}")


def random_mix(count: int, seed: int = 7, extent: float = 4.0, with_ground: bool = True) -> Scene:
    """A small random heap of boxes, spheres, capsules and hulls in a cube of side `extent`,
    overlapping freely (narrowphase coverage for every shape pair)."""
    rng = np.random.default_rng(seed)
    bodies = R.body_defaults(count)
    bodies["position"] = rng.uniform(-extent / 2, extent / 2, size=(count, 3)).astype(np.float32)
    bodies["position"][:, 1] += extent / 2 + 0.6
    bodies["orientation"] = uniform_quaternions(rng, count)
    bodies["velocity"] = rng.normal(0, 0.5, size=(count, 3)).astype(np.float32)
    bodies["angular_velocity"] = rng.normal(0, 0.5, size=(count, 3)).astype(np.float32)
    bodies["density"] = 1000.0
    colliders = R.collider_defaults(count)
    kinds = rng.choice([R.SHAPE_CUBOID, R.SHAPE_SPHERE, R.SHAPE_CAPSULE, R.SHAPE_HULL], size=count)
    colliders["shape"] = kinds
    colliders["half_extents"] = rng.uniform(0.2, 0.6, size=(count, 3)).astype(np.float32)
    colliders["radius"] = rng.uniform(0.2, 0.5, size=count).astype(np.float32)
    colliders["half_height"] = rng.uniform(0.1, 0.4, size=count).astype(np.float32)
    colliders["restitution"] = 0.1
    hulls = []
    for row in np.nonzero(kinds == R.SHAPE_HULL)[0]:
        m = int(rng.integers(8, 33))
        d = rng.normal(size=(m, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        hulls.append((d * rng.uniform(0.3, 0.6)).astype(np.float32))
        colliders["source"][row] = len(hulls) - 1
    if with_ground:
        bodies, colliders = _ground(bodies, colliders, 0.0, 0.5, 0.1)
    return Scene(bodies, colliders, hulls, f"random_mix_{count}")


def hanging_chains(chains_x: int = 64, chains_z: int = 64, links: int = 32, seed: int = 2, spacing: float = 1.5,
                   ground: float = -10.0, spin: float = 0.5) -> Scene:
    """chains_x x chains_z chains of `links` boxes (half-extents 0.1 x 0.25 x 0.1 m, density 1000)
    joined end to end by ball joints (anchors at +-0.25 m on y), each hanging from a static anchor
    body on a grid at `spacing` metres and y = 0; every box starts with an angular velocity drawn
    from N(0, spin) rad/s per axis, and the chains swing into each other and onto a ground plane at
    y = `ground`. 64 x 64 x 32 gives 131,072 boxes and 131,072 joints."""
    rng = np.random.default_rng(seed)
    chains = chains_x * chains_z
    n = chains * links
    ci, ck = np.meshgrid(np.arange(chains_x), np.arange(chains_z), indexing="ij")
    top = np.stack([(ci.ravel() - (chains_x - 1) / 2) * spacing, np.zeros(chains),
                    (ck.ravel() - (chains_z - 1) / 2) * spacing], axis=1)
    link = np.arange(links)
    pos = top[:, None, :] + np.stack([np.zeros(links), -0.25 - 0.5 * link, np.zeros(links)], axis=1)[None, :, :]
    bodies = R.body_defaults(n)
    bodies["position"] = pos.reshape(n, 3).astype(np.float32)
    bodies["angular_velocity"] = rng.normal(0.0, spin, size=(n, 3)).astype(np.float32)
    bodies["density"] = 1000.0
    colliders = R.collider_defaults(n)
    colliders["shape"] = R.SHAPE_CUBOID
    colliders["half_extents"] = (0.1, 0.25, 0.1)
    colliders["friction"] = 0.5
    anchors = R.body_defaults(chains)
    anchors["position"] = top.astype(np.float32)
    anchors["mass"] = 0.0
    anchors["collider_first"] = n + np.arange(chains)
    anchor_colliders = R.collider_defaults(chains)
    anchor_colliders["radius"] = 0.05
    bodies = np.concatenate([bodies, anchors])
    colliders = np.concatenate([colliders, anchor_colliders])
    joints = np.zeros(n, JOINT)
    chain = np.repeat(np.arange(chains), links)
    k = np.tile(link, chains)
    joints["first"] = np.where(k == 0, n + chain, np.arange(n) - 1)
    joints["second"] = np.arange(n)
    joints["anchor_a"] = np.where((k == 0)[:, None], np.zeros(3), np.array([0.0, -0.25, 0.0]))
    joints["anchor_b"] = (0.0, 0.25, 0.0)
    bodies, colliders = _ground(bodies, colliders, ground, 0.5, 0.0)
    return Scene(bodies, colliders, [], f"hanging_chains_{n}", joints)


def batch(parts: list) -> Scene:
    """Independent scenes as sub-worlds of one batch: body i of part w is in sub-world w."""
    bodies, colliders, hulls, joints, worlds = [], [], [], [], []
    body_base = collider_base = 0
    for index, part in enumerate(parts):
        b = part.bodies.copy()
        c = part.colliders.copy()
        b["collider_first"] += collider_base
        hull = c["shape"] == R.SHAPE_HULL
        c["source"][hull] += len(hulls)
        hulls.extend(part.hulls)
        if part.joints is not None:
            j = part.joints.copy()
            j["first"] += body_base
            j["second"] += body_base
            joints.append(j)
        bodies.append(b)
        colliders.append(c)
        worlds.append(np.full(len(b), index, np.uint32))
        body_base += len(b)
        collider_base += len(c)
    return Scene(np.concatenate(bodies), np.concatenate(colliders), hulls, f"batch_{len(parts)}",
                 np.concatenate(joints) if joints else None, np.concatenate(worlds))


def box_lattice(count: int, seed: int, spacing: float = 1.1) -> Scene:
    """`count` unit cubes (falling_boxes' shape mix and distributions) on the smallest cubic lattice
    that holds them, above their own ground plane."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(count ** (1.0 / 3.0) - 1e-9))
    idx = np.arange(count)
    i, j, k = idx % side, (idx // side) % side, idx // (side * side)
    base = np.stack([(i - (side - 1) / 2) * spacing, 0.6 + j * spacing, (k - (side - 1) / 2) * spacing], axis=1)
    bodies = R.body_defaults(count)
    bodies["position"] = (base + rng.uniform(-0.05, 0.05, size=(count, 3))).astype(np.float32)
    bodies["orientation"] = yaw_quaternions(rng.uniform(0.0, 2 * np.pi, count))
    bodies["density"] = 1000.0
    colliders = R.collider_defaults(count)
    colliders["shape"] = R.SHAPE_CUBOID
    colliders["half_extents"] = 0.5
    colliders["friction"] = 0.5
    colliders["restitution"] = 0.0
    bodies, colliders = _ground(bodies, colliders, 0.0, 0.5, 0.0)
    return Scene(bodies, colliders, [], f"box_lattice_{count}")


def batched_world_parts(worlds: int = 4096, seed: int = 4, smallest: int = 16, largest: int = 2048) -> list:
    """`worlds` independent box lattices, each on its own ground plane, whose body counts are drawn
    log-uniform in [smallest, largest]."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(smallest), np.log(largest), worlds)).astype(np.int64)
    return [box_lattice(int(n), seed * 100003 + w) for w, n in enumerate(counts)]


def batched_worlds(worlds: int = 4096, seed: int = 4) -> Scene:
    """batched_world_parts as one batch (one sub-world each); 4,096 worlds hold about 1.76M bodies."""
    return batch(batched_world_parts(worlds, seed))


def tower_world(seed: int, levels: int = 8, footprint: int = 4, distance: float = 4.0, box_mass: float = 1.0,
                friction: float = 0.5, heading: float | None = None, gap: float = 0.0) -> Scene:
    """An `levels`-high tower of unit boxes (half-extent 0.5 m) on a `footprint` x `footprint` base,
    standing on a ground plane, and a sphere of radius 0.5 m resting on the ground `distance` metres
    from the tower's axis, on a heading drawn from U(-0.2, 0.2) rad about -x (or the given heading).
    Every collider has the given friction; boxes and sphere the given mass. Neighbouring columns stand
    `gap` metres apart (0: face to face). The sphere is the last body before the plane."""
    rng = np.random.default_rng(seed)
    n = levels * footprint * footprint
    i, k, j = np.meshgrid(np.arange(footprint), np.arange(footprint), np.arange(levels), indexing="ij")
    pitch = 1.0 + gap
    pos = np.stack([(i.ravel() - (footprint - 1) / 2) * pitch, 0.5 + j.ravel(), (k.ravel() - (footprint - 1) / 2) * pitch],
                   axis=1)
    order = np.lexsort((pos[:, 2], pos[:, 0], pos[:, 1]))  # level by level
    bodies = R.body_defaults(n + 1)
    bodies["position"][:n] = pos[order].astype(np.float32)
    drawn = rng.uniform(-0.2, 0.2)
    heading = drawn if heading is None else heading
    bodies["position"][n] = (-distance * np.cos(heading), 0.5, -distance * np.sin(heading))
    bodies["mass"] = box_mass
    bodies["collider_first"] = np.arange(n + 1)
    colliders = R.collider_defaults(n + 1)
    colliders["shape"][:n] = R.SHAPE_CUBOID
    colliders["half_extents"][:n] = 0.5
    colliders["shape"][n] = R.SHAPE_SPHERE
    colliders["radius"][n] = 0.5
    colliders["friction"] = friction
    colliders["restitution"] = 0.0
    bodies, colliders = _ground(bodies, colliders, 0.0, friction, 0.0)
    return Scene(bodies, colliders, [], f"tower_{n}")


def sphere_launches(scene: Scene, states: np.ndarray, rows: np.ndarray, seed: int = 5) -> np.ndarray:
    """Launch velocities of the spheres at body rows `rows` (states in row order): a speed drawn from
    U(3, 8) m/s toward the vertical axis of the sphere's own world (x = z = 0)."""
    rng = np.random.default_rng(seed + 7919)
    direction = -states["position"][rows].astype(np.float64)
    direction[:, 1] = 0.0
    direction /= np.linalg.norm(direction, axis=1, keepdims=True)
    return (direction * rng.uniform(3.0, 8.0, len(rows))[:, None]).astype(np.float32)


def differentiable_towers(worlds: int = 256, seed: int = 5, levels: int = 8, footprint: int = 4) -> Scene:
    """`worlds` tower worlds (tower_world) as one batch: per-body masses drawn from U(0.5, 2) kg and a
    per-world friction from U(0.3, 0.8), every collider of a world (its plane included) at the
    world's friction."""
    rng = np.random.default_rng(seed)
    parts = []
    for w in range(worlds):
        part = tower_world(seed * 1000003 + w, levels, footprint, friction=float(rng.uniform(0.3, 0.8)))
        part.bodies["mass"][:-1] = rng.uniform(0.5, 2.0, len(part.bodies) - 1).astype(np.float32)
        parts.append(part)
    scene = batch(parts)
    scene.name = f"differentiable_towers_{worlds}"
    return scene


WORKLOADS = {
    "falling_boxes_1000": lambda: falling_boxes(seed=0),
    "mixed_pile_32768": lambda: mixed_pile(side=32, seed=1),
    "mixed_pile_262144": lambda: mixed_pile(side=64, seed=1),
    "hanging_chains_8192": lambda: hanging_chains(16, 16, 32),
    "hanging_chains_131072": lambda: hanging_chains(64, 64, 32),
    "batched_worlds_256": lambda: batched_worlds(256),
    "batched_worlds_4096": lambda: batched_worlds(4096),
    "differentiable_towers_256": lambda: differentiable_towers(256),
}
