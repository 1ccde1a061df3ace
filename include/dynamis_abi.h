/*
 * dynamis_abi.h - byte-exact record layouts and constants of the Dynamis rigid-body ABI.
 *
 * These are the data contract the drop-in boundary keeps: the same bytes the reference's
 * `dynamis-abi` crate passes between its Rust host and its WGSL passes. Every struct mirrors a
 * WGSL storage layout in crates/dynamis-abi/abi/records.wgsl (vec3f aligned to 16 bytes, sized
 * 12), so a Rust caller can hand over `bytemuck` slices of its `*Record` types unchanged.
 *
 * Plain C (C99 / C++), no CUDA or torch types. Offsets are asserted at the bottom.
 */
#ifndef DYNAMIS_ABI_H
#define DYNAMIS_ABI_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- constants: crates/dynamis-abi/src/constant.rs:6-127, records.wgsl:1 ---- */
#define DYN_CONTACT_MAX_POINTS 4u
#define DYN_BODY_KINEMATIC 1u
#define DYN_BODY_CCD 2u
#define DYN_OVERRIDE_SLEEP_LINEAR 4u
#define DYN_OVERRIDE_SLEEP_ANGULAR 8u
#define DYN_NO_COLLISION_FILTER 0xFFFFFFFFu
#define DYN_SOLVER_DELTA_WORDS 8u
#define DYN_SHAPE_NONE 0u
#define DYN_SHAPE_SPHERE 1u
#define DYN_SHAPE_CUBOID 2u
#define DYN_SHAPE_CAPSULE 3u
#define DYN_SHAPE_CYLINDER 4u
#define DYN_SHAPE_HULL 5u
#define DYN_SHAPE_MESH 6u
#define DYN_SHAPE_HEIGHTFIELD 7u
#define DYN_SHAPE_TRIANGLE 8u
#define DYN_SHAPE_PLANE 9u
#define DYN_COLLIDER_SENSOR 1u
#define DYN_EVENT_MODE_BEGIN_END 2u
#define DYN_EVENT_MODE_PERSIST 4u
#define DYN_CONTACT_ANNOUNCED 0x80000000u
#define DYN_ISLAND_WAKE 1u
#define DYN_FEATURE_POINT 0u
#define DYN_FEATURE_VERTEX (1u << 28)
#define DYN_FEATURE_EDGE (2u << 28)
#define DYN_FEATURE_FACE (3u << 28)
#define DYN_FEATURE_KIND_MASK 0xF0000000u
#define DYN_FEATURE_FIELD_BITS 14u
#define DYN_FEATURE_FIELD_MASK ((1u << 14) - 1u)
#define DYN_FEATURE_INDEX_LIMIT (1u << 12)
#define DYN_FEATURE_CLIP (1u << 12)
#define DYN_FEATURE_FACE_BIT (1u << 13)
#define DYN_MAX_CELLS_PER_AXIS 2u
#define DYN_MAX_CELLS_PER_COLLIDER 8u
#define DYN_ENTRY_INDEX_BITS 24u
#define DYN_ENTRY_INDEX_MASK ((1u << 24) - 1u)
#define DYN_ENTRY_CELL_SHIFT 24u
#define DYN_ENTRY_CELL_MASK (7u << 24)
#define DYN_ENTRY_KIND_SHIFT 27u
#define DYN_ENTRY_KIND_MASK (3u << 27)
#define DYN_ENTRY_MOBILE (1u << 29)
#define DYN_ENTRY_AWAKE (1u << 30)
#define DYN_ENTRY_PRIMARY (1u << 31)
#define DYN_ENTRY_KIND_COLLIDER 0u
#define DYN_LEVEL_KEY_SHIFT 27u
#define DYN_CELL_HASH_MASK 0x07FFFFFFu
#define DYN_GRID_LEVEL_LIMIT 30u
/* body edit kinds and patch masks: crates/dynamis-abi/src/constant.rs:6-18 */
#define DYN_EDIT_PATCH 0u
#define DYN_EDIT_FORCE 1u
#define DYN_EDIT_TORQUE 2u
#define DYN_EDIT_IMPULSE 3u
#define DYN_EDIT_SLEEP 4u
#define DYN_EDIT_WAKE 5u
#define DYN_EDIT_FORCE_AT_POINT 6u
#define DYN_EDIT_IMPULSE_AT_POINT 7u
#define DYN_EDIT_ANGULAR_IMPULSE 8u
#define DYN_PATCH_POSITION 1u
#define DYN_PATCH_VELOCITY 2u
#define DYN_PATCH_ORIENTATION 4u
#define DYN_PATCH_ANGULAR_VELOCITY 8u
/* constraint kinds and flags: crates/dynamis-abi/src/constant.rs:88-103 */
#define DYN_CONSTRAINT_BALL 0u
#define DYN_CONSTRAINT_DISTANCE 1u
#define DYN_CONSTRAINT_REVOLUTE 2u
#define DYN_CONSTRAINT_PRISMATIC 3u
#define DYN_CONSTRAINT_FIXED 4u
#define DYN_CONSTRAINT_GEAR 5u
#define DYN_CONSTRAINT_PULLEY 6u
#define DYN_CONSTRAINT_CONE 7u
#define DYN_CONSTRAINT_SIXDOF 8u
#define DYN_CONSTRAINT_DISABLE_COLLISIONS 1u
#define DYN_CONSTRAINT_HAS_LIMIT 2u
#define DYN_CONSTRAINT_HAS_MOTOR 4u
#define DYN_CONSTRAINT_IS_SPRING 8u
#define DYN_CONSTRAINT_HAS_SWING 16u
#define DYN_CONSTRAINT_HAS_BREAK 32u
#define DYN_CONSTRAINT_WARM_START 64u
#define DYN_CONSTRAINT_ACCUMULATOR_SLOTS 16u
#define DYN_NO_BODY 0xFFFFFFFFu
#define DYN_NO_SLOT 0xFFFFFFFFu
#define DYN_NO_SURFACE 0xFFFFFFFFu
#define DYN_NO_TRIANGLE 0xFFFFFFFFu
/* crates/dynamis-abi/src/constant.rs:272-274 */
#define DYN_SOLVER_VELOCITY_SCALE 262144.0f
#define DYN_SOLVER_POSITION_SCALE 16777216.0f

/* ---- device counters: crates/dynamis-abi/src/counter.rs:76-128 (slot = declaration order) ---- */
enum dyn_counter {
    DYN_COUNTER_ENTRIES = 0,
    DYN_COUNTER_RESTING_ENTRIES = 1,
    DYN_COUNTER_RESTING_LEVELS = 2,
    DYN_COUNTER_RESTING_REBUILD = 3,
    DYN_COUNTER_RESTING_SORT = 4,
    DYN_COUNTER_AWAKE_BASE = 5,
    DYN_COUNTER_IMMOVABLE_ENTRIES = 6,
    DYN_COUNTER_IMMOVABLE_EMITTED = 7,
    DYN_COUNTER_IMMOVABLE_LEVELS = 8,
    DYN_COUNTER_ENTRY_BASE = 9,
    DYN_COUNTER_PAIRS = 10,
    DYN_COUNTER_GRID_LEVELS = 11,
    DYN_COUNTER_CONTACTS = 12,
    DYN_COUNTER_ARCHIVED = 13,
    DYN_COUNTER_JOINTS = 14,
    DYN_COUNTER_EVENTS = 15,
    DYN_COUNTER_REFUSED_PAIRS = 16,
    DYN_COUNTER_REFUSED_EVENTS = 17,
    DYN_COUNTER_ENTRY_FAULTS = 18,
    DYN_COUNTER_RESTING = 19,
    DYN_COUNTER_REFUSED_RESTING = 20,
    DYN_COUNTER_SLEPT = 21,
    DYN_COUNTER_WOKE = 22,
    DYN_COUNTER_ACTIVE = 23,
    DYN_COUNTER_WOKE_DEFERRED = 24,
    DYN_COUNTER_RESTING_GATHER = 25,
    DYN_COUNTER_RESTING_INDEX = 26,
    DYN_COUNTER_RESTING_PENDING = 27,
    DYN_COUNTER_ISLANDS = 28,
    DYN_COUNTER_ISLAND_FAULTS = 29,
    DYN_COUNTER_BLOCKS = 30,
    DYN_COUNTER_SOLVER_ROWS = 31,
    DYN_COUNTER_SOLVE_LINEAR_RESIDUAL = 32,
    DYN_COUNTER_SOLVE_ANGULAR_RESIDUAL = 33,
    DYN_COUNTER_COARSE_ACTIVE = 34,
    DYN_COUNTER_GRID_SCALE = 35,
    DYN_COUNTER_GRID_EXTENT = 36,
    DYN_COUNTER_BREAKS = 37,
    DYN_COUNTER_PARTICLE_REACH = 38,
    DYN_COUNTER_COARSE_NEIGHBOURS = 39,
    DYN_COUNTER_LIVE = 40,
    DYN_COUNTER_LIVE_FAULTS = 41,
    DYN_COUNTER_ROW_FAULTS = 42,
    DYN_COUNTER_SOFT_ACTIVE = 43,
    DYN_COUNTER_SOFT_SLEPT = 44,
    DYN_COUNTER_SOFT_WOKE = 45,
    DYN_COUNTER_REFUSED_CONTACTS = 46,
    DYN_COUNTER_STEP = 47,
    DYN_COUNTER_IMPACTS = 48,
    DYN_COUNTER_REFUSED_IMPACTS = 49,
    DYN_COUNTER_SOFT_EVENTS = 50,
    DYN_COUNTER_REFUSED_SOFT_EVENTS = 51,
    DYN_COUNTER_DEVICE_COUNT = 52
};

/* ---- records: crates/dynamis-abi/abi/records.wgsl ---- */

/* records.wgsl:8-47 (176 bytes) */
typedef struct dyn_step_params {
    float gravity[4];
    float dt;
    float substep_dt;
    float damping;
    float angular_damping;
    uint32_t body_count;
    uint32_t substeps;
    uint32_t solve_iterations;
    uint32_t constraint_count;
    float relaxation;
    float slop;
    float restitution_threshold;
    float max_velocity;
    float max_angular_velocity;
    uint32_t dynamic_count;
    float sleep_velocity;
    float sleep_angular_velocity;
    float sleep_time;
    uint32_t friction_combine;
    uint32_t restitution_combine;
    uint32_t position_iterations;
    float contact_margin;
    uint32_t collider_count;
    uint32_t soft_iterations;
    uint32_t soft_substeps;
    uint32_t particle_count;
    uint32_t element_count;
    float soft_substep_dt;
    uint32_t soft_body_count;
    uint32_t attachment_count;
    float settle_velocity;
    uint32_t observed_count;
    uint32_t observed_joint_count;
    uint32_t character_count;
    uint32_t vehicle_count;
    uint32_t vehicle_wheel_count;
    uint32_t wake_all;
    uint32_t field_count;
    uint32_t _pad_tail[3];
} dyn_step_params;

/* records.wgsl:145-164 (144 bytes) */
typedef struct dyn_body_state_record {
    float position[3];
    float _pad0;
    float prev_position[3];
    float _pad1;
    float prev_orientation[4];
    float orientation[4];
    float velocity[3];
    float _pad2;
    float angular_velocity[3];
    float _pad3;
    float force[3];
    float _pad4;
    float torque[3];
    float _pad5;
    uint32_t body_id;
    uint32_t generation;
    float sleep_timer;
    uint32_t sleeping;
} dyn_body_state_record;

/* records.wgsl:166-184 (128 bytes) */
typedef struct dyn_body_descriptor_record {
    float inverse_mass;
    float linear_damping;
    float angular_damping;
    float gravity_scale;
    float sleep_velocity;
    float sleep_angular_velocity;
    uint32_t flags;
    uint32_t _pad0;
    uint32_t collision_group;
    uint32_t collision_mask;
    uint32_t _pad1;
    uint32_t _pad4;
    float com[3];
    float _pad2;
    float inertia[6];
    float inverse_inertia[6];
    float _pad3[4];
} dyn_body_descriptor_record;

/* records.wgsl:208-228 (112 bytes) */
typedef struct dyn_collider_record {
    uint32_t slot;
    uint32_t kind;
    uint32_t flags;
    float radius;
    float half_height;
    float relaxation;
    float damping_ratio;
    float impact_force;
    float half_extents[3];
    uint32_t collision_group;
    float local_offset[3];
    uint32_t collision_mask;
    float local_rotation[4];
    float friction;
    float restitution;
    uint32_t source;
    float rolling_friction;
    float scale[3];
    float spin_friction;
} dyn_collider_record;

/* records.wgsl:256-273 (80 bytes) */
typedef struct dyn_shape_source_record {
    uint32_t kind;
    uint32_t vertex_offset;
    uint32_t vertex_count;
    uint32_t triangle_offset;
    uint32_t node_offset;
    uint32_t node_count;
    uint32_t cell_offset;
    uint32_t cell_count;
    uint32_t grid_rows;
    uint32_t grid_cols;
    uint32_t _pad0;
    uint32_t _pad1;
    float local_min[3];
    float _pad2;
    float local_max[3];
    float _pad3;
} dyn_shape_source_record;

/* records.wgsl:299-304 (32 bytes) */
typedef struct dyn_aabb_record {
    float min[3];
    float _pad0;
    float max[3];
    float _pad1;
} dyn_aabb_record;

/* records.wgsl:306-311 (32 bytes) */
typedef struct dyn_grid_entry_record {
    float min[3];
    uint32_t group;
    float max[3];
    uint32_t info;
} dyn_grid_entry_record;

/* records.wgsl:313-322 (64 bytes) */
typedef struct dyn_manifold_point_record {
    float position[3];
    float depth;
    float local_a[3];
    float _pad0;
    float local_b[3];
    float accumulated_normal;
    float accumulated_tangent_1;
    float accumulated_tangent_2;
    uint32_t feature;
    uint32_t _pad1;
} dyn_manifold_point_record;

/* records.wgsl:331-353 (352 bytes) */
typedef struct dyn_contact_record {
    uint32_t a;
    uint32_t b;
    uint32_t point_count;
    uint32_t sensor;
    uint32_t first_body_id;
    uint32_t second_body_id;
    uint32_t first_generation;
    uint32_t second_generation;
    float normal[3];
    uint32_t events;
    uint32_t surface;
    uint32_t triangle;
    float friction;
    float restitution;
    float rolling_friction;
    float spin_friction;
    float carried_normal;
    float carried_tangent;
    float relaxation;
    float damping_ratio;
    uint32_t _pad0[2];
    dyn_manifold_point_record points[4];
} dyn_contact_record;

/* records.wgsl:355-416 (400 bytes by WGSL storage layout: 11 vec3f fields before cone_angle, 14 after) */
typedef struct dyn_constraint_descriptor_record {
    uint32_t kind;
    uint32_t first_body_id;
    uint32_t second_body_id;
    uint32_t flags;
    float anchor_a[3];
    float _pad1;
    float anchor_b[3];
    float _pad2;
    float axis_a[3];
    float _pad3;
    float axis_b[3];
    float _pad4;
    float distance;
    float limit_min;
    float limit_max;
    float swing_a;
    float swing_b;
    float motor_speed;
    float motor_max_force;
    float spring_frequency;
    float spring_damping_ratio;
    float break_force;
    float break_torque;
    float gear_ratio;
    float pulley_fixed_a[3];
    float _pad_pulley_a;
    float pulley_fixed_b[3];
    float _pad_pulley_b;
    float motor_position;
    float motor_stiffness;
    float motor_damping;
    float cone_angle;
    float linear_limit_min[4];
    float linear_limit_max[4];
    float angular_limit_min[4];
    float angular_limit_max[4];
    float linear_motor_speed[4];
    float linear_motor_position[4];
    float linear_motor_stiffness[4];
    float linear_motor_damping[4];
    float linear_motor_force[4];
    float angular_motor_speed[4];
    float angular_motor_position[4];
    float angular_motor_stiffness[4];
    float angular_motor_damping[4];
    float angular_motor_force[4];
} dyn_constraint_descriptor_record;

/* records.wgsl:193-199 (160 bytes): one command for one body, applied at the next step */
typedef struct dyn_body_edit_record {
    uint32_t kind;  /* DYN_EDIT_* */
    uint32_t mask;  /* DYN_PATCH_* for DYN_EDIT_PATCH */
    uint32_t _pad0;
    uint32_t _pad1;
    dyn_body_state_record state;  /* the values the edit carries (see body_edits.wgsl) */
} dyn_body_edit_record;

/* records.wgsl:201-206 (16 bytes): the edits [first, first + len) of one row */
typedef struct dyn_body_edit_run_record {
    uint32_t row;
    uint32_t first;
    uint32_t len;
    uint32_t _pad;
} dyn_body_edit_run_record;

/* records.wgsl:440-443 (8 bytes) */
typedef struct dyn_constraint_rows_record {
    uint32_t first_row;
    uint32_t second_row;
} dyn_constraint_rows_record;

/* records.wgsl:445-454 (64 bytes) */
typedef struct dyn_constraint_reaction_record {
    float linear_first[3];
    float _pad_linear_first;
    float angular_first[3];
    float _pad_angular_first;
    float linear_second[3];
    float _pad_linear_second;
    float angular_second[3];
    float _pad_angular_second;
} dyn_constraint_reaction_record;

/* records.wgsl:418-426 (160 bytes) */
typedef struct dyn_constraint_runtime_record {
    dyn_constraint_reaction_record reaction;
    float reference[4];
    float accumulated[DYN_CONSTRAINT_ACCUMULATOR_SLOTS];
    uint32_t broken;
    uint32_t constraint_id;
    uint32_t generation;
    uint32_t _pad0;
} dyn_constraint_runtime_record;

/* Scene queries: crates/dynamis-abi/src/constant.rs:84-120 (query kinds, targets, filter flags),
 * records.wgsl:5 (QUERY_CANDIDATES) */
#define DYN_QUERY_RAY 0u
#define DYN_QUERY_SPHERE 1u
#define DYN_QUERY_CUBOID 2u
#define DYN_QUERY_SWEEP 3u
#define DYN_QUERY_POINT 4u
#define DYN_QUERY_CONVEX 5u
#define DYN_QUERY_TARGET_COLLIDERS 1u
#define DYN_QUERY_TARGET_PARTICLES 2u
#define DYN_FILTER_IGNORE_SENSORS 1u
#define DYN_FILTER_IGNORE_SLEEPING 2u
#define DYN_FILTER_IGNORE_STATIC 4u
#define DYN_FILTER_IGNORE_KINEMATIC 8u
#define DYN_QUERY_CANDIDATES 4096u

/* records.wgsl:456-469 (48 bytes) */
typedef struct dyn_query_filter_record {
    uint32_t flags;    /* DYN_FILTER_* */
    uint32_t targets;  /* DYN_QUERY_TARGET_* */
    uint32_t group;    /* 0: no group filter */
    uint32_t mask;
    uint32_t exclude_id;  /* DYN_NO_BODY: none */
    uint32_t exclude_generation;
    uint32_t include_id;  /* DYN_NO_BODY: none */
    uint32_t include_generation;
    uint32_t exclude_soft_id;
    uint32_t exclude_soft_generation;
    uint32_t include_soft_id;
    uint32_t include_soft_generation;
} dyn_query_filter_record;

/* records.wgsl:471-488 (144 bytes): QueryRecord. count and overflow are written back. */
typedef struct dyn_query_record {
    uint32_t kind;        /* DYN_QUERY_* */
    uint32_t shape_kind;  /* the probe's DYN_SHAPE_* (sphere, cuboid, capsule, cylinder, hull) */
    uint32_t source;      /* the probe's hull source */
    uint32_t max_hits;
    dyn_query_filter_record filters;
    float origin[3];
    float _pad0;
    float direction[3];
    float extent;         /* ray length, sphere radius, sweep length */
    float radius;
    float half_height;
    uint32_t count;       /* hits written */
    uint32_t hit_base;    /* first hit slot of this query in the batch's hit array */
    float half_extents[3];
    uint32_t overflow;    /* 1: more hits existed than were written */
    float orientation[4];
} dyn_query_record;

/* records.wgsl:490-499 (48 bytes): QueryHit */
typedef struct dyn_query_hit_record {
    uint32_t body_id;
    uint32_t body_generation;
    float distance;
    uint32_t scene_target;  /* the candidate: kind << DYN_ENTRY_KIND_SHIFT | collider slot */
    float point[3];
    uint32_t triangle;
    float normal[3];
    uint32_t surface;
} dyn_query_hit_record;

#ifdef __cplusplus
} /* extern "C" */
#endif

/* Offsets pinned by crates/dynamis-abi/tests/records.rs:241-276 and build.rs:90-170. */
#ifdef __cplusplus
#define DYN_ABI_ASSERT(c, m) static_assert(c, m)
#else
#define DYN_ABI_ASSERT(c, m) _Static_assert(c, m)
#endif
DYN_ABI_ASSERT(sizeof(dyn_step_params) == 176, "StepParams is 176 bytes");
DYN_ABI_ASSERT(sizeof(dyn_body_state_record) == 144, "BodyState is 144 bytes");
DYN_ABI_ASSERT(offsetof(dyn_body_state_record, velocity) == 64, "BodyState.velocity @64");
DYN_ABI_ASSERT(offsetof(dyn_body_state_record, body_id) == 128, "BodyState.body_id @128");
DYN_ABI_ASSERT(sizeof(dyn_body_descriptor_record) == 128, "BodyDescriptor is 128 bytes");
DYN_ABI_ASSERT(offsetof(dyn_body_descriptor_record, com) == 48, "BodyDescriptor.com @48");
DYN_ABI_ASSERT(offsetof(dyn_body_descriptor_record, inertia) == 64, "BodyDescriptor.inertia @64");
DYN_ABI_ASSERT(offsetof(dyn_body_descriptor_record, inverse_inertia) == 88, "inverse_inertia @88");
DYN_ABI_ASSERT(sizeof(dyn_collider_record) == 112, "Collider is 112 bytes");
DYN_ABI_ASSERT(offsetof(dyn_collider_record, relaxation) == 20, "Collider.relaxation @20");
DYN_ABI_ASSERT(offsetof(dyn_collider_record, half_extents) == 32, "Collider.half_extents @32");
DYN_ABI_ASSERT(offsetof(dyn_collider_record, collision_group) == 44, "Collider.collision_group @44");
DYN_ABI_ASSERT(offsetof(dyn_collider_record, local_offset) == 48, "Collider.local_offset @48");
DYN_ABI_ASSERT(offsetof(dyn_collider_record, collision_mask) == 60, "Collider.collision_mask @60");
DYN_ABI_ASSERT(offsetof(dyn_collider_record, local_rotation) == 64, "Collider.local_rotation @64");
DYN_ABI_ASSERT(offsetof(dyn_collider_record, friction) == 80, "Collider.friction @80");
DYN_ABI_ASSERT(offsetof(dyn_collider_record, scale) == 96, "Collider.scale @96");
DYN_ABI_ASSERT(offsetof(dyn_collider_record, spin_friction) == 108, "Collider.spin_friction @108");
DYN_ABI_ASSERT(sizeof(dyn_shape_source_record) == 80, "ShapeSource is 80 bytes");
DYN_ABI_ASSERT(sizeof(dyn_aabb_record) == 32, "Aabb is 32 bytes");
DYN_ABI_ASSERT(sizeof(dyn_grid_entry_record) == 32, "GridEntry is 32 bytes");
DYN_ABI_ASSERT(sizeof(dyn_manifold_point_record) == 64, "ManifoldPoint is 64 bytes");
DYN_ABI_ASSERT(offsetof(dyn_manifold_point_record, accumulated_normal) == 44, "ManifoldPoint.accumulated_normal @44");
DYN_ABI_ASSERT(offsetof(dyn_manifold_point_record, feature) == 56, "ManifoldPoint.feature @56");
DYN_ABI_ASSERT(sizeof(dyn_contact_record) == 352, "Contact is 352 bytes");
DYN_ABI_ASSERT(offsetof(dyn_contact_record, normal) == 32, "Contact.normal @32");
DYN_ABI_ASSERT(offsetof(dyn_contact_record, events) == 44, "Contact.events @44");
DYN_ABI_ASSERT(offsetof(dyn_contact_record, carried_normal) == 72, "Contact.carried_normal @72");
DYN_ABI_ASSERT(offsetof(dyn_contact_record, carried_tangent) == 76, "Contact.carried_tangent @76");
DYN_ABI_ASSERT(offsetof(dyn_contact_record, relaxation) == 80, "Contact.relaxation @80");
DYN_ABI_ASSERT(offsetof(dyn_contact_record, damping_ratio) == 84, "Contact.damping_ratio @84");
DYN_ABI_ASSERT(offsetof(dyn_contact_record, points) == 96, "Contact.points @96");
DYN_ABI_ASSERT(sizeof(dyn_constraint_descriptor_record) == 400, "ConstraintDescriptor is 400 bytes");
DYN_ABI_ASSERT(sizeof(dyn_constraint_rows_record) == 8, "ConstraintRows is 8 bytes");
DYN_ABI_ASSERT(sizeof(dyn_constraint_reaction_record) == 64, "ConstraintReaction is 64 bytes");
DYN_ABI_ASSERT(sizeof(dyn_body_edit_record) == 160, "BodyEdit is 160 bytes");
DYN_ABI_ASSERT(offsetof(dyn_body_edit_record, state) == 16, "BodyEdit.state @16");
DYN_ABI_ASSERT(sizeof(dyn_body_edit_run_record) == 16, "BodyEditRun is 16 bytes");
DYN_ABI_ASSERT(sizeof(dyn_constraint_runtime_record) == 160, "ConstraintRuntime is 160 bytes");
DYN_ABI_ASSERT(offsetof(dyn_constraint_runtime_record, accumulated) == 80, "ConstraintRuntime.accumulated @80");
DYN_ABI_ASSERT(offsetof(dyn_constraint_runtime_record, broken) == 144, "ConstraintRuntime.broken @144");
DYN_ABI_ASSERT(offsetof(dyn_constraint_descriptor_record, axis_a) == 48, "ConstraintDescriptor.axis_a @48");
DYN_ABI_ASSERT(offsetof(dyn_constraint_descriptor_record, break_force) == 116, "ConstraintDescriptor.break_force @116");
DYN_ABI_ASSERT(sizeof(dyn_query_filter_record) == 48, "QueryFilter is 48 bytes");
DYN_ABI_ASSERT(sizeof(dyn_query_record) == 144, "Query is 144 bytes");
DYN_ABI_ASSERT(offsetof(dyn_query_record, origin) == 64, "Query.origin @64");
DYN_ABI_ASSERT(offsetof(dyn_query_record, extent) == 92, "Query.extent @92");
DYN_ABI_ASSERT(offsetof(dyn_query_record, hit_base) == 108, "Query.hit_base @108");
DYN_ABI_ASSERT(offsetof(dyn_query_record, overflow) == 124, "Query.overflow @124");
DYN_ABI_ASSERT(offsetof(dyn_query_record, orientation) == 128, "Query.orientation @128");
DYN_ABI_ASSERT(sizeof(dyn_query_hit_record) == 48, "QueryHit is 48 bytes");
DYN_ABI_ASSERT(offsetof(dyn_query_hit_record, normal) == 32, "QueryHit.normal @32");

#endif /* DYNAMIS_ABI_H */
