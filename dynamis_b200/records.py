"""numpy views of the byte-exact Dynamis ABI records (include/dynamis_abi.h).

Each dtype reproduces a WGSL storage layout of crates/dynamis-abi/abi/records.wgsl, so arrays of
these records can be handed to the C ABI by pointer and compared field by field in tests.
"""
from __future__ import annotations

import numpy as np

COUNTER_DEVICE_COUNT = 52
COUNTERS = [
    "ENTRIES", "RESTING_ENTRIES", "RESTING_LEVELS", "RESTING_REBUILD", "RESTING_SORT", "AWAKE_BASE",
    "IMMOVABLE_ENTRIES", "IMMOVABLE_EMITTED", "IMMOVABLE_LEVELS", "ENTRY_BASE", "PAIRS", "GRID_LEVELS",
    "CONTACTS", "ARCHIVED", "JOINTS", "EVENTS", "REFUSED_PAIRS", "REFUSED_EVENTS", "ENTRY_FAULTS",
    "RESTING", "REFUSED_RESTING", "SLEPT", "WOKE", "ACTIVE", "WOKE_DEFERRED", "RESTING_GATHER",
    "RESTING_INDEX", "RESTING_PENDING", "ISLANDS", "ISLAND_FAULTS", "BLOCKS", "SOLVER_ROWS",
    "SOLVE_LINEAR_RESIDUAL", "SOLVE_ANGULAR_RESIDUAL", "COARSE_ACTIVE", "GRID_SCALE", "GRID_EXTENT",
    "BREAKS", "PARTICLE_REACH", "COARSE_NEIGHBOURS", "LIVE", "LIVE_FAULTS", "ROW_FAULTS", "SOFT_ACTIVE",
    "SOFT_SLEPT", "SOFT_WOKE", "REFUSED_CONTACTS", "STEP", "IMPACTS", "REFUSED_IMPACTS", "SOFT_EVENTS",
    "REFUSED_SOFT_EVENTS",
]
COUNTER = {name: slot for slot, name in enumerate(COUNTERS)}

SHAPE_SPHERE, SHAPE_CUBOID, SHAPE_CAPSULE, SHAPE_CYLINDER, SHAPE_HULL, SHAPE_PLANE = 1, 2, 3, 4, 5, 9
NO_BODY = 0xFFFFFFFF
NO_COLLISION_FILTER = 0xFFFFFFFF
CONTACT_ANNOUNCED = 0x80000000
BODY_KINEMATIC = 1  # BodyDescriptorRecord flags (constant.rs)
BODY_CCD = 2
SOLVER_GUARD_ROW_MASS = 1  # dyn_set_solver_guard


def _dtype(fields, size):
    names = [f[0] for f in fields]
    formats = [f[1] for f in fields]
    offsets = [f[2] for f in fields]
    return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": size})


STEP_PARAMS = np.dtype([
    ("gravity", "<f4", 4), ("dt", "<f4"), ("substep_dt", "<f4"), ("damping", "<f4"), ("angular_damping", "<f4"),
    ("body_count", "<u4"), ("substeps", "<u4"), ("solve_iterations", "<u4"), ("constraint_count", "<u4"),
    ("relaxation", "<f4"), ("slop", "<f4"), ("restitution_threshold", "<f4"), ("max_velocity", "<f4"),
    ("max_angular_velocity", "<f4"), ("dynamic_count", "<u4"), ("sleep_velocity", "<f4"),
    ("sleep_angular_velocity", "<f4"), ("sleep_time", "<f4"), ("friction_combine", "<u4"),
    ("restitution_combine", "<u4"), ("position_iterations", "<u4"), ("contact_margin", "<f4"),
    ("collider_count", "<u4"), ("soft_iterations", "<u4"), ("soft_substeps", "<u4"), ("particle_count", "<u4"),
    ("element_count", "<u4"), ("soft_substep_dt", "<f4"), ("soft_body_count", "<u4"), ("attachment_count", "<u4"),
    ("settle_velocity", "<f4"), ("observed_count", "<u4"), ("observed_joint_count", "<u4"),
    ("character_count", "<u4"), ("vehicle_count", "<u4"), ("vehicle_wheel_count", "<u4"), ("wake_all", "<u4"),
    ("field_count", "<u4"), ("_pad_tail", "<u4", 3),
])



def _fields(spec):
    return [(name, (fmt, shape) if shape > 1 else fmt, off) for name, fmt, shape, off in spec]


BODY_STATE = _dtype(_fields([
    ("position", "<f4", 3, 0), ("prev_position", "<f4", 3, 16), ("prev_orientation", "<f4", 4, 32),
    ("orientation", "<f4", 4, 48), ("velocity", "<f4", 3, 64), ("angular_velocity", "<f4", 3, 80),
    ("force", "<f4", 3, 96), ("torque", "<f4", 3, 112), ("body_id", "<u4", 1, 128), ("generation", "<u4", 1, 132),
    ("sleep_timer", "<f4", 1, 136), ("sleeping", "<u4", 1, 140),
]), 144)

BODY_DESCRIPTOR = _dtype(_fields([
    ("inverse_mass", "<f4", 1, 0), ("linear_damping", "<f4", 1, 4), ("angular_damping", "<f4", 1, 8),
    ("gravity_scale", "<f4", 1, 12), ("sleep_velocity", "<f4", 1, 16), ("sleep_angular_velocity", "<f4", 1, 20),
    ("flags", "<u4", 1, 24), ("collision_group", "<u4", 1, 32), ("collision_mask", "<u4", 1, 36),
    ("com", "<f4", 3, 48), ("inertia", "<f4", 6, 64), ("inverse_inertia", "<f4", 6, 88),
]), 128)

COLLIDER = _dtype(_fields([
    ("slot", "<u4", 1, 0), ("kind", "<u4", 1, 4), ("flags", "<u4", 1, 8), ("radius", "<f4", 1, 12),
    ("half_height", "<f4", 1, 16), ("relaxation", "<f4", 1, 20), ("damping_ratio", "<f4", 1, 24),
    ("impact_force", "<f4", 1, 28), ("half_extents", "<f4", 3, 32), ("collision_group", "<u4", 1, 44),
    ("local_offset", "<f4", 3, 48), ("collision_mask", "<u4", 1, 60), ("local_rotation", "<f4", 4, 64),
    ("friction", "<f4", 1, 80), ("restitution", "<f4", 1, 84), ("source", "<u4", 1, 88),
    ("rolling_friction", "<f4", 1, 92), ("scale", "<f4", 3, 96), ("spin_friction", "<f4", 1, 108),
]), 112)

SHAPE_SOURCE = _dtype(_fields([
    ("kind", "<u4", 1, 0), ("vertex_offset", "<u4", 1, 4), ("vertex_count", "<u4", 1, 8),
    ("triangle_offset", "<u4", 1, 12), ("node_offset", "<u4", 1, 16), ("node_count", "<u4", 1, 20),
    ("local_min", "<f4", 3, 48), ("local_max", "<f4", 3, 64),
]), 80)

AABB = _dtype(_fields([("min", "<f4", 3, 0), ("max", "<f4", 3, 16)]), 32)

MANIFOLD_POINT = _dtype(_fields([
    ("position", "<f4", 3, 0), ("depth", "<f4", 1, 12), ("local_a", "<f4", 3, 16), ("local_b", "<f4", 3, 32),
    ("accumulated_normal", "<f4", 1, 44), ("accumulated_tangent_1", "<f4", 1, 48),
    ("accumulated_tangent_2", "<f4", 1, 52), ("feature", "<u4", 1, 56),
]), 64)

CONTACT = _dtype([
    ("a", "<u4", 0), ("b", "<u4", 4), ("point_count", "<u4", 8), ("sensor", "<u4", 12),
    ("first_body_id", "<u4", 16), ("second_body_id", "<u4", 20), ("first_generation", "<u4", 24),
    ("second_generation", "<u4", 28), ("normal", ("<f4", 3), 32), ("events", "<u4", 44), ("surface", "<u4", 48),
    ("triangle", "<u4", 52), ("friction", "<f4", 56), ("restitution", "<f4", 60), ("rolling_friction", "<f4", 64),
    ("spin_friction", "<f4", 68), ("carried_normal", "<f4", 72), ("carried_tangent", "<f4", 76),
    ("relaxation", "<f4", 80), ("damping_ratio", "<f4", 84), ("points", (MANIFOLD_POINT, 4), 96),
], 352)

# records.wgsl:355-416 (the fields this path uses; the rest of the 400 bytes are kept as raw padding)
CONSTRAINT_DESCRIPTOR = _dtype(_fields([
    ("kind", "<u4", 1, 0), ("first_body_id", "<u4", 1, 4), ("second_body_id", "<u4", 1, 8), ("flags", "<u4", 1, 12),
    ("anchor_a", "<f4", 3, 16), ("anchor_b", "<f4", 3, 32), ("axis_a", "<f4", 3, 48), ("axis_b", "<f4", 3, 64),
    ("distance", "<f4", 1, 80), ("limit_min", "<f4", 1, 84), ("limit_max", "<f4", 1, 88), ("swing_a", "<f4", 1, 92),
    ("swing_b", "<f4", 1, 96), ("break_force", "<f4", 1, 116), ("break_torque", "<f4", 1, 120),
    ("gear_ratio", "<f4", 1, 124),
]), 400)
CONSTRAINT_ROWS = _dtype(_fields([("first_row", "<u4", 1, 0), ("second_row", "<u4", 1, 4)]), 8)
# records.wgsl:418-426 with ConstraintReaction :445-454
CONSTRAINT_RUNTIME = _dtype(_fields([
    ("linear_first", "<f4", 3, 0), ("angular_first", "<f4", 3, 16), ("linear_second", "<f4", 3, 32),
    ("angular_second", "<f4", 3, 48), ("reference", "<f4", 4, 64), ("accumulated", "<f4", 16, 80),
    ("broken", "<u4", 1, 144), ("constraint_id", "<u4", 1, 148), ("generation", "<u4", 1, 152),
]), 160)
CONSTRAINT_BALL = 0
# records.wgsl BodyEdit: a command kind, a patch mask and the state it carries (160 bytes)
# scene queries (records.wgsl:456-499; constant.rs:84-120)
QUERY_RAY, QUERY_SPHERE, QUERY_CUBOID, QUERY_SWEEP, QUERY_POINT, QUERY_CONVEX = 0, 1, 2, 3, 4, 5
QUERY_TARGET_COLLIDERS, QUERY_TARGET_PARTICLES = 1, 2
FILTER_IGNORE_SENSORS, FILTER_IGNORE_SLEEPING, FILTER_IGNORE_STATIC, FILTER_IGNORE_KINEMATIC = 1, 2, 4, 8
QUERY_CANDIDATES = 4096
NO_TRIANGLE = 0xFFFFFFFF
QUERY_FILTER = np.dtype([(name, "<u4") for name in (
    "flags", "targets", "group", "mask", "exclude_id", "exclude_generation", "include_id", "include_generation",
    "exclude_soft_id", "exclude_soft_generation", "include_soft_id", "include_soft_generation")])
QUERY = _dtype(_fields([
    ("kind", "<u4", 1, 0), ("shape_kind", "<u4", 1, 4), ("source", "<u4", 1, 8), ("max_hits", "<u4", 1, 12),
]) + [("filters", QUERY_FILTER, 16)] + _fields([
    ("origin", "<f4", 3, 64), ("direction", "<f4", 3, 80), ("extent", "<f4", 1, 92), ("radius", "<f4", 1, 96),
    ("half_height", "<f4", 1, 100), ("count", "<u4", 1, 104), ("hit_base", "<u4", 1, 108),
    ("half_extents", "<f4", 3, 112), ("overflow", "<u4", 1, 124), ("orientation", "<f4", 4, 128),
]), 144)
QUERY_HIT = _dtype(_fields([
    ("body_id", "<u4", 1, 0), ("body_generation", "<u4", 1, 4), ("distance", "<f4", 1, 8), ("scene_target", "<u4", 1, 12),
    ("point", "<f4", 3, 16), ("triangle", "<u4", 1, 28), ("normal", "<f4", 3, 32), ("surface", "<u4", 1, 44),
]), 48)
assert QUERY_FILTER.itemsize == 48 and QUERY.itemsize == 144 and QUERY_HIT.itemsize == 48


def query_filter(max_hits: int = 4, group: int = 0, mask: int = 0xFFFFFFFF, ignore_sensors: bool = True,
                 ignore_sleeping: bool = False, ignore_static: bool = False, ignore_kinematic: bool = False,
                 exclude=None, include=None, colliders: bool = True, particles: bool = True) -> dict:
    """QueryFilter::default (crates/dynamis-model/src/query.rs:41-58) with overrides; exclude and
    include are (body id, generation) pairs."""
    return dict(max_hits=max_hits, group=group, mask=mask, ignore_sensors=ignore_sensors,
                ignore_sleeping=ignore_sleeping, ignore_static=ignore_static, ignore_kinematic=ignore_kinematic,
                exclude=exclude, include=include, colliders=colliders, particles=particles)


def _query_record(kind: int, filt: dict | None) -> np.ndarray:
    """query_record (crates/dynamis-abi/src/query.rs:44-74)."""
    f = query_filter() if filt is None else filt
    q = np.zeros(1, QUERY)
    q["kind"] = kind
    flags = ((FILTER_IGNORE_SENSORS if f["ignore_sensors"] else 0) | (FILTER_IGNORE_SLEEPING if f["ignore_sleeping"] else 0)
             | (FILTER_IGNORE_STATIC if f["ignore_static"] else 0) | (FILTER_IGNORE_KINEMATIC if f["ignore_kinematic"] else 0))
    fr = q["filters"]
    fr["flags"] = flags
    fr["targets"] = (QUERY_TARGET_COLLIDERS if f["colliders"] else 0) | (QUERY_TARGET_PARTICLES if f["particles"] else 0)
    fr["group"], fr["mask"] = f["group"], f["mask"]
    fr["exclude_id"], fr["exclude_generation"] = f["exclude"] if f["exclude"] is not None else (NO_BODY, 0)
    fr["include_id"], fr["include_generation"] = f["include"] if f["include"] is not None else (NO_BODY, 0)
    fr["exclude_soft_id"] = fr["include_soft_id"] = NO_BODY
    q["filters"] = fr
    q["max_hits"] = f["max_hits"]
    return q


def _probe_shape(q: np.ndarray, shape: dict) -> None:
    """shape_fields (query.rs:76-98): shape = dict(kind=SHAPE_*, radius, half_height, half_extents, source)."""
    q["shape_kind"] = shape["kind"]
    q["source"] = shape.get("source", 0)
    q["radius"] = shape.get("radius", 0.0)
    q["half_height"] = shape.get("half_height", 0.0)
    q["half_extents"] = shape.get("half_extents", (0.0, 0.0, 0.0))


def ray_query(origin, direction, max_t: float, filt: dict | None = None) -> np.ndarray:
    q = _query_record(QUERY_RAY, filt)
    q["origin"], q["direction"], q["extent"] = origin, direction, max_t
    return q


def sphere_query(center, radius: float, filt: dict | None = None) -> np.ndarray:
    q = _query_record(QUERY_SPHERE, filt)
    q["shape_kind"], q["origin"], q["extent"], q["radius"] = SHAPE_SPHERE, center, radius, radius
    return q


def point_query(origin, filt: dict | None = None) -> np.ndarray:
    q = _query_record(QUERY_POINT, filt)
    q["shape_kind"], q["origin"] = SHAPE_SPHERE, origin
    return q


def cuboid_query(center, half_extents, filt: dict | None = None) -> np.ndarray:
    q = _query_record(QUERY_CUBOID, filt)
    q["shape_kind"], q["origin"], q["half_extents"] = SHAPE_CUBOID, center, half_extents
    return q


def overlap_query(shape: dict, orientation, position, filt: dict | None = None) -> np.ndarray:
    q = _query_record(QUERY_CONVEX, filt)
    q["origin"], q["orientation"] = position, orientation
    _probe_shape(q, shape)
    return q


def sweep_query(shape: dict, orientation, start, direction, length: float, filt: dict | None = None) -> np.ndarray:
    q = _query_record(QUERY_SWEEP, filt)
    q["origin"], q["direction"], q["extent"], q["orientation"] = start, direction, length, orientation
    _probe_shape(q, shape)
    return q


BODY_EDIT = np.dtype({"names": ["kind", "mask", "state"], "formats": ["<u4", "<u4", BODY_STATE],
                      "offsets": [0, 4, 16], "itemsize": 160})
EDIT_PATCH, EDIT_FORCE, EDIT_TORQUE, EDIT_IMPULSE, EDIT_SLEEP, EDIT_WAKE = 0, 1, 2, 3, 4, 5
EDIT_FORCE_AT_POINT, EDIT_IMPULSE_AT_POINT, EDIT_ANGULAR_IMPULSE = 6, 7, 8
PATCH_POSITION, PATCH_VELOCITY, PATCH_ORIENTATION, PATCH_ANGULAR_VELOCITY = 1, 2, 4, 8
CONSTRAINT_DISABLE_COLLISIONS, CONSTRAINT_HAS_BREAK, CONSTRAINT_WARM_START = 1, 32, 64

# C ABI descriptors (include/dynamis_cuda.h)
CONFIG = np.dtype([
    ("gravity", "<f4", 3), ("damping", "<f4"), ("angular_damping", "<f4"), ("substeps", "<u4"),
    ("solve_iterations", "<u4"), ("position_iterations", "<u4"), ("relaxation", "<f4"), ("slop", "<f4"),
    ("contact_margin", "<f4"), ("restitution_threshold", "<f4"), ("max_velocity", "<f4"),
    ("max_angular_velocity", "<f4"), ("sleep_velocity", "<f4"), ("sleep_angular_velocity", "<f4"),
    ("sleep_time", "<f4"), ("friction_combine", "<u4"), ("restitution_combine", "<u4"),
])
CAPACITY = np.dtype([("bodies", "<u4"), ("colliders", "<u4"), ("pairs", "<u4"), ("contacts", "<u4")])
LAUNCH_CONFIG = np.dtype([("grid_blocks_per_sm", "<u4"), ("solve_threads", "<u4"), ("gjk_blocks_per_sm", "<u4"),
                          ("epa_blocks_per_sm", "<u4")])
COLLIDER_DESC = np.dtype([
    ("shape", "<u4"), ("radius", "<f4"), ("half_height", "<f4"), ("half_extents", "<f4", 3), ("source", "<u4"),
    ("offset", "<f4", 3), ("rotation", "<f4", 4), ("scale", "<f4", 3), ("friction", "<f4"),
    ("restitution", "<f4"), ("rolling_friction", "<f4"), ("spin_friction", "<f4"), ("contact_frequency", "<f4"),
    ("contact_damping_ratio", "<f4"), ("sensor", "<u4"), ("events", "<u4"), ("collision_group", "<u4"),
    ("collision_mask", "<u4"), ("impact_force", "<f4"),
])
BODY_DESC = np.dtype([
    ("position", "<f4", 3), ("orientation", "<f4", 4), ("velocity", "<f4", 3), ("angular_velocity", "<f4", 3),
    ("mass", "<f4"), ("density", "<f4"), ("gravity_scale", "<f4"), ("linear_damping", "<f4"),
    ("angular_damping", "<f4"), ("sleep_velocity", "<f4"), ("sleep_angular_velocity", "<f4"),
    ("collision_group", "<u4"), ("collision_mask", "<u4"), ("kinematic", "<u4"), ("ccd", "<u4"),
    ("collider_first", "<u4"), ("collider_count", "<u4"),
])

assert STEP_PARAMS.itemsize == 176 and BODY_STATE.itemsize == 144 and BODY_DESCRIPTOR.itemsize == 128
# dynamis_cuda.h dyn_body_grad: d loss / d one body row's state (64 bytes)
BODY_GRAD = _dtype(_fields([
    ("position", "<f4", 3, 0), ("orientation", "<f4", 4, 16), ("velocity", "<f4", 3, 32),
    ("angular_velocity", "<f4", 3, 48),
]), 64)

assert COLLIDER.itemsize == 112 and SHAPE_SOURCE.itemsize == 80 and CONTACT.itemsize == 352
assert MANIFOLD_POINT.itemsize == 64 and AABB.itemsize == 32
assert CONSTRAINT_DESCRIPTOR.itemsize == 400 and CONSTRAINT_ROWS.itemsize == 8 and CONSTRAINT_RUNTIME.itemsize == 160


def collider_defaults(n: int) -> np.ndarray:
    """ColliderDesc::new defaults (crates/dynamis-model/src/collider.rs:52-70) for n colliders."""
    c = np.zeros(n, COLLIDER_DESC)
    c["shape"] = SHAPE_SPHERE
    c["radius"] = 0.5
    c["rotation"][:, 3] = 1.0
    c["scale"] = 1.0
    c["friction"] = 0.5
    c["contact_frequency"] = np.inf
    c["contact_damping_ratio"] = 1.0
    c["collision_group"] = NO_COLLISION_FILTER
    c["collision_mask"] = NO_COLLISION_FILTER
    c["impact_force"] = np.inf
    return c


def body_defaults(n: int) -> np.ndarray:
    """BodyDesc::new defaults (crates/dynamis-model/src/body.rs:174-194) for n bodies."""
    b = np.zeros(n, BODY_DESC)
    b["orientation"][:, 3] = 1.0
    b["mass"] = 1.0
    b["gravity_scale"] = 1.0
    b["linear_damping"] = -1.0
    b["angular_damping"] = -1.0
    b["sleep_velocity"] = -1.0
    b["sleep_angular_velocity"] = -1.0
    b["collision_group"] = 1
    b["collision_mask"] = 0xFFFFFFFF
    b["collider_count"] = 1
    b["collider_first"] = np.arange(n, dtype=np.uint32)
    return b


def body_edit(kind: int, mask: int = 0, position=None, orientation=None, velocity=None, angular_velocity=None,
              force=None, torque=None) -> np.ndarray:
    """One BodyEdit record (command.rs BodyCommand::edit): `velocity` carries an impulse, `position`
    a point of application or a patched position, `angular_velocity` an angular impulse."""
    e = np.zeros(1, BODY_EDIT)
    e["kind"], e["mask"] = kind, mask
    st = e["state"]
    for name, value in (("position", position), ("orientation", orientation), ("velocity", velocity),
                        ("angular_velocity", angular_velocity), ("force", force), ("torque", torque)):
        if value is not None:
            st[name] = value
    e["state"] = st
    return e
