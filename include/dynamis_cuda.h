/*
 * dynamis_cuda.h - C ABI of the B200 rigid-body step (libdynamis_cuda.so).
 *
 * This is the drop-in boundary for the reference's `dynamis-world` step path. Each entry point
 * names the Rust API it replaces (paths relative to the reference project). Records crossing the
 * boundary are the byte-exact ABI layouts of dynamis_abi.h. All memory is owned by the library
 * behind the opaque world handle; every call returns a dyn_status (0 = ok) and never aborts.
 * One world is used from one host thread at a time; distinct worlds are independent.
 *
 * Host-only calls (configuration, hulls, spawning, record export) work without a GPU; the device
 * is touched on the first call that needs it (step, upload, download, debug reads).
 */
#ifndef DYNAMIS_CUDA_H
#define DYNAMIS_CUDA_H

#include <stdint.h>

#include "dynamis_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define DYN_API __attribute__((visibility("default")))
#else
#define DYN_API
#endif

typedef int32_t dyn_status;
#define DYN_OK 0
#define DYN_ERR_INVALID 1         /* argument or scene the reference would refuse (it panics) */
#define DYN_ERR_CAPACITY 2        /* a declared capacity is too small for the scene */
#define DYN_ERR_CUDA 3            /* a CUDA runtime call failed; see dyn_last_error */
#define DYN_ERR_NO_DEVICE 4       /* no CUDA device, or the requested ordinal does not exist */
#define DYN_ERR_DEVICE_STATUS 5   /* a kernel gave up a bounded wait; see dyn_device_status */
#define DYN_ERR_DEGENERATE 6      /* a hull point set spans no volume */
#define DYN_NOT_READY 7           /* no observation has completed yet (dyn_try_state, dyn_try_counters) */

typedef struct dyn_world dyn_world;

/* PhysicsConfig: crates/dynamis-model/src/config.rs:12-100 (defaults from dyn_config_default). */
typedef struct dyn_config {
    float gravity[3];
    float damping;
    float angular_damping;
    uint32_t substeps;
    uint32_t solve_iterations;
    uint32_t position_iterations;
    float relaxation;
    float slop;
    float contact_margin;
    float restitution_threshold;
    float max_velocity;
    float max_angular_velocity;
    float sleep_velocity;
    float sleep_angular_velocity;
    float sleep_time;
    uint32_t friction_combine;    /* 0 multiply, 1 min, 2 max, 3 average (param.rs:160-167) */
    uint32_t restitution_combine;
} dyn_config;

/* Stream capacities, fixed up front (the reference grows streams from lagged counters:
 * crates/dynamis-broadphase/src/capacity.rs:27-78). Zero means "size from the scene". */
typedef struct dyn_capacity {
    uint32_t bodies;
    uint32_t colliders;
    uint32_t pairs;
    uint32_t contacts;
} dyn_capacity;

/* ColliderDesc: crates/dynamis-model/src/collider.rs (one collider of a body). */
typedef struct dyn_collider_desc {
    uint32_t shape;          /* DYN_SHAPE_SPHERE, _CUBOID, _CAPSULE, _CYLINDER, _HULL, _PLANE */
    float radius;            /* sphere, capsule, cylinder */
    float half_height;       /* capsule, cylinder */
    float half_extents[3];   /* cuboid */
    uint32_t source;         /* hull source from dyn_add_hull */
    float offset[3];
    float rotation[4];
    float scale[3];
    float friction;          /* default 0.5 */
    float restitution;       /* default 0 */
    float rolling_friction;
    float spin_friction;
    float contact_frequency; /* +inf = hard contact (relaxation 0) */
    float contact_damping_ratio; /* default 1 */
    uint32_t sensor;
    uint32_t events;         /* DYN_EVENT_MODE_* bits */
    uint32_t collision_group; /* DYN_NO_COLLISION_FILTER = inherit the body's */
    uint32_t collision_mask;
    float impact_force;      /* +inf = none */
} dyn_collider_desc;

/* BodyDesc: crates/dynamis-model/src/body.rs:88-200. A body owns colliders
 * [collider_first, collider_first + collider_count) of the collider array passed beside it. */
typedef struct dyn_body_desc {
    float position[3];
    float orientation[4];
    float velocity[3];
    float angular_velocity[3];
    float mass;              /* used when density <= 0; 0 makes a static body */
    float density;           /* > 0: mass = density x solid volume */
    float gravity_scale;     /* default 1 */
    float linear_damping;    /* < 0 = the config's damping */
    float angular_damping;   /* < 0 = the config's angular damping */
    float sleep_velocity;    /* < 0 = the config's threshold */
    float sleep_angular_velocity;
    uint32_t collision_group; /* default 1 */
    uint32_t collision_mask;  /* default all */
    uint32_t kinematic;
    uint32_t ccd;
    uint32_t collider_first;
    uint32_t collider_count;
} dyn_body_desc;

DYN_API uint32_t dyn_abi_version(void);
DYN_API const char* dyn_status_string(dyn_status status);

/* PhysicsConfig::default (config.rs:76-100), ColliderDesc::new and BodyDesc::new defaults. */
DYN_API void dyn_config_default(dyn_config* out);
DYN_API void dyn_collider_desc_default(dyn_collider_desc* out);
DYN_API void dyn_body_desc_default(dyn_body_desc* out);

/* World::new (crates/dynamis-world/src/lib.rs:86). device = CUDA ordinal used by device calls. */
DYN_API dyn_status dyn_world_create(const dyn_config* config, const dyn_capacity* capacity, int32_t device,
                                    dyn_world** out);
DYN_API dyn_status dyn_world_destroy(dyn_world* world);
/* Last error text of this world (empty when none). */
DYN_API const char* dyn_last_error(const dyn_world* world);
/* Run device work on a caller-owned cudaStream_t (NULL = the world's own stream). */
DYN_API dyn_status dyn_world_set_stream(dyn_world* world, void* cuda_stream);

/* World::add_hull_from_mesh (crates/dynamis-world/src/shape.rs:50-56): the convex hull of the
 * vertices (xyz triples) the triangles (index triples) reference, built as dynamis-hull's hull()
 * builds it (crates/dynamis-hull/src/hull.rs:53-288: its vertices numbered by first appearance over
 * the surviving faces), with the solid integrals of solid.rs:62-105, becomes a hull shape source. */
DYN_API dyn_status dyn_add_hull_from_mesh(dyn_world* world, const float* xyz, uint32_t nv, const uint32_t* triangles,
                                          uint32_t nt, uint32_t* out_source);
/* dyn_add_hull_from_mesh of n points all counted as referenced (a point cloud). */
DYN_API dyn_status dyn_add_hull(dyn_world* world, const float* xyz, uint32_t n, uint32_t* out_source);
/* World::add_hull (crates/dynamis-world/src/shape.rs:24-26): a hull given as its own vertices and
 * outward triangles, kept as given. */
DYN_API dyn_status dyn_add_hull_mesh(dyn_world* world, const float* xyz, uint32_t nv, const uint32_t* triangles, uint32_t nt,
                                     uint32_t* out_source);
DYN_API dyn_status dyn_hull_info(const dyn_world* world, uint32_t source, uint32_t* vertex_count,
                                 uint32_t* triangle_count, float* volume, float centroid[3]);

/* World::spawn (crates/dynamis-world/src/body.rs:108-130) for n bodies at once: builds
 * BodyStateRecord::initial, BodyDescriptorRecord::build (mass properties of
 * crates/dynamis-model/src/mass.rs:155-212) and ColliderRecord::build. out_ids[i] = body id. */
DYN_API dyn_status dyn_spawn_bodies(dyn_world* world, const dyn_body_desc* bodies, uint32_t n,
                                    const dyn_collider_desc* colliders, uint32_t k, uint32_t* out_ids);

/* Replaces the scene with ready-made ABI records (the Rust shim passes its bytemuck slices).
 * Rows must hold the dynamic bodies first (the reference's row census); owners[i] is the body row
 * of collider i. Shape sources come from dyn_add_hull on this world. */
DYN_API dyn_status dyn_upload_bodies(dyn_world* world, const dyn_body_state_record* states,
                                     const dyn_body_descriptor_record* descs, uint32_t n,
                                     const dyn_collider_record* colliders, const uint32_t* owners, uint32_t k);
/* Overwrites the n body states (row order) of the current scene. */
DYN_API dyn_status dyn_upload_states(dyn_world* world, const dyn_body_state_record* states, uint32_t n);

/* The device's pair and contact stream capacities (0 before the first step). The pair stream
 * widens by itself, before a later dyn_step, once a step refused pairs or needed more than half of
 * it: to twice the demand, at least twice its size (replaces World::stream_capacity,
 * crates/dynamis-world/src/lib.rs:132, and the widening of
 * crates/dynamis-broadphase/src/capacity.rs:27-80). */
DYN_API dyn_status dyn_stream_capacity(const dyn_world* world, uint32_t* pairs, uint32_t* contacts);

/* Host copy of the scene as rows: sizes, then records (any output pointer may be NULL). */
DYN_API dyn_status dyn_scene_sizes(const dyn_world* world, uint32_t* bodies, uint32_t* dynamic_bodies,
                                   uint32_t* colliders, uint32_t* sources, uint32_t* vertices);
DYN_API dyn_status dyn_export_scene(const dyn_world* world, dyn_body_state_record* states,
                                    dyn_body_descriptor_record* descs, dyn_collider_record* colliders,
                                    uint32_t* owners, dyn_shape_source_record* sources, float* vertices_xyzw);
/* StepParamsRecord::new (crates/dynamis-abi/src/param.rs:110-158) for this scene and dt. */
DYN_API dyn_status dyn_step_params_for(const dyn_world* world, float dt, dyn_step_params* out);

/* World::step (crates/dynamis-world/src/step.rs:34-39): enqueues one step (a CUDA graph launch)
 * and returns without waiting, as the reference's submit does. */
DYN_API dyn_status dyn_step(dyn_world* world, float dt);
/* World::wait (observation.rs:484): blocks until queued steps finish; reports the sticky device
 * status (DYN_ERR_DEVICE_STATUS when a kernel's bounded wait ran out). */
DYN_API dyn_status dyn_sync(dyn_world* world);
DYN_API dyn_status dyn_device_status(dyn_world* world, uint32_t* status);

/* World::read_state (body.rs:326) for all rows, and one body by id. Synchronises. */
DYN_API dyn_status dyn_download_states(dyn_world* world, dyn_body_state_record* out, uint32_t n);
DYN_API dyn_status dyn_read_state(dyn_world* world, uint32_t body_id, dyn_body_state_record* out);
/* World::measured (readback.rs:215): the device counters, slots of dynamis_abi.h's dyn_counter. */
DYN_API dyn_status dyn_read_counters(dyn_world* world, uint32_t* out, uint32_t n);

/* Parity hooks: the last step's intermediate products (synchronise). count = items available. */
DYN_API dyn_status dyn_debug_aabbs(dyn_world* world, dyn_aabb_record* out, uint32_t cap, uint32_t* count);
DYN_API dyn_status dyn_debug_entries(dyn_world* world, uint32_t* keys, uint32_t* infos, uint32_t cap, uint32_t* count);
DYN_API dyn_status dyn_debug_pairs(dyn_world* world, uint32_t* major, uint32_t* minor, uint32_t cap, uint32_t* count);
DYN_API dyn_status dyn_debug_contacts(dyn_world* world, dyn_contact_record* out, uint32_t cap, uint32_t* count);
DYN_API dyn_status dyn_debug_islands(dyn_world* world, uint32_t* out, uint32_t cap, uint32_t* count);
/* Scene queries: World::ray_query, sphere_query, cuboid_query, point_query, overlap_query and
 * sweep_query, then resolve_queries and query_hits (crates/dynamis-world/src/query.rs:50-175;
 * scene_cast.wgsl), as one synchronous call against the world's current body states. Each record
 * is a QueryRecord as crates/dynamis-abi/src/query.rs:103-181 builds it (kind, probe shape, filters,
 * origin, direction, extent, max_hits). The library gives query i the hit slots
 * [hit_base, hit_base + min(max_hits, DYN_QUERY_CANDIDATES)) in submission order (hit_capacity must
 * hold their sum, else DYN_ERR_CAPACITY), writes its hits nearest first, and sets count and overflow
 * (1 when more hits existed than were written, or the candidate walk passed DYN_QUERY_CANDIDATES).
 * Targets are colliders (particles belong to soft bodies, outside this library). The call rebuilds
 * the grid index from the current states first, as the reference's query run does, so
 * dyn_read_counters then shows that index's ENTRIES and GRID_* counters. Refused (DYN_ERR_INVALID)
 * for an invalid record and for a world of batched sub-worlds. */
DYN_API dyn_status dyn_query(dyn_world* world, dyn_query_record* queries, uint32_t n, dyn_query_hit_record* hits,
                             uint32_t hit_capacity);
/* The triangles of a hull source: index triples over its vertices (dyn_hull_info's numbering). */
DYN_API dyn_status dyn_hull_triangles(const dyn_world* world, uint32_t source, uint32_t* out, uint32_t cap, uint32_t* count);

/* The frozen contacts the next step reads (freeze_contacts.wgsl / thaw_contacts.wgsl: contacts of
 * body pairs that were both at rest when a step ended), six words each: first body id, its
 * generation, second body id, its generation, collider a, collider b. Order is not meaningful.
 * The reference reads them through World::inspect_contacts with its live contacts. */
DYN_API dyn_status dyn_debug_resting(dyn_world* world, uint32_t* out, uint32_t cap, uint32_t* count);

/* Per-stage timing (World::gpu_pass_timings, step.rs:187-190). With timing on, dyn_step runs the
 * stages eagerly with CUDA events between them instead of the graph; dyn_stage_timings returns
 * the last step's milliseconds per stage and their names. */
DYN_API dyn_status dyn_set_timing(dyn_world* world, int32_t enabled);
/* Kernel launches in one step (kernel nodes of the captured step graph; 0 before the first step). */
DYN_API uint32_t dyn_step_kernel_count(const dyn_world* world);
DYN_API uint32_t dyn_stage_count(void);
DYN_API const char* dyn_stage_name(uint32_t stage);
DYN_API dyn_status dyn_stage_timings(dyn_world* world, float* ms, uint32_t n);

/* Standalone operator (crates/dynamis-sort/src/radix.rs:397 RadixSort::sort): stable LSD sort of
 * n device-resident (major, minor) u32 keys with an optional u32 payload, minor_digits of the
 * minor word then major_digits of the major word (8-bit digits). Pointers are device pointers;
 * minor/payload may be NULL. Uses the world's stream and scratch. */
DYN_API dyn_status dyn_radix_sort(dyn_world* world, uint32_t* major, uint32_t* minor, uint32_t* payload, uint32_t n,
                                  uint32_t major_digits, uint32_t minor_digits);

/* ---- body commands ----
 * World's body commands (set_position / set_velocity / apply_force / apply_impulse / sleep / wake ...,
 * compiled to BodyEditRecords by crates/dynamis-world/src/command.rs:129-184): edits[i] applies to
 * the body with id body_ids[i]. Edits queue on the host and run at the start of the next dyn_step,
 * after the step clears forces and before anything reads the bodies (body_edits.wgsl), in the order
 * given for each body. */
/* Lagged observations (World::observe_bodies / observe_all_bodies / stop_observing_all_bodies / poll /
 * try_state, crates/dynamis-world/src/observation.rs:480-516; the counter ring of
 * dynamis-gpu/src/readback.rs:158-173). While observing, every dyn_step also copies, on the world's
 * stream, the observed bodies' state records and the counters into one of four pinned host slots.
 * dyn_try_state and dyn_try_counters read the newest slot whose copy has completed, with the step
 * number it was taken after, and never wait for the GPU: DYN_NOT_READY until a first copy
 * completes. When every slot is still in flight, a step's copy replaces the oldest one (the newest
 * observation wins); nothing waits.
 * body_ids == NULL observes every body (bodies spawned later included); otherwise the ids are added
 * to the observed set. */
DYN_API dyn_status dyn_observe_bodies(dyn_world* world, const uint32_t* body_ids, uint32_t n);
DYN_API dyn_status dyn_stop_observing(dyn_world* world);
DYN_API dyn_status dyn_poll(dyn_world* world);
DYN_API dyn_status dyn_try_state(dyn_world* world, uint32_t body_id, dyn_body_state_record* out, uint64_t* step);
DYN_API dyn_status dyn_try_counters(dyn_world* world, uint32_t* out, uint32_t n, uint64_t* step);

/* World::remove (crates/dynamis-world/src/body.rs:132-155) for n bodies at once. The bodies and
 * their colliders leave the world at the next dyn_step; the other bodies keep their simulated
 * states (the device's states are read back first), and body ids are not reused. Refused with
 * DYN_ERR_INVALID when an id is unknown, repeated or already removed, or while a constraint still
 * names the body (the reference asserts the body is unreferenced), and for worlds whose scene came
 * from dyn_upload_bodies. A removal re-uploads the scene, so the next step starts without
 * archived contacts (no warm start for that one step). */
DYN_API dyn_status dyn_remove_bodies(dyn_world* world, const uint32_t* body_ids, uint32_t n);

DYN_API dyn_status dyn_edit_bodies(dyn_world* world, const uint32_t* body_ids, const dyn_body_edit_record* edits, uint32_t n);

/* ---- batched worlds ----
 * Thousands of independent worlds stepped by one dyn_step: every body id gets a sub-world
 * (world_of_body[id], n = the number of bodies spawned or uploaded), and bodies of different
 * sub-worlds never pair, contact or join an island, so each sub-world steps exactly as it would
 * alone. Sub-world 0 is the default. No counterpart in the reference, which steps one world per
 * World::step; this is the batched-worlds configuration of the benchmark. */
DYN_API dyn_status dyn_set_body_worlds(dyn_world* world, const uint32_t* world_of_body, uint32_t n);
/* The sub-world of every row (dyn_export_scene's row order), for a checker. */
DYN_API dyn_status dyn_export_body_worlds(const dyn_world* world, uint32_t* rows_out);

/* ---- constraints: ball joints (row a11 of the path) ----
 * World::add_constraint(first, second, ConstraintDesc::ball(anchor_a, anchor_b))
 * (crates/dynamis-world/src/constraint.rs:121, crates/dynamis-model/src/constraint.rs:568): a ball joint
 * between two bodies by id, anchors in each body's frame, with the reference's defaults (collisions
 * between the two bodies disabled, warm start on, axis +y). *out_id is the constraint id (creation
 * order). The joint takes effect at the next dyn_step. */
DYN_API dyn_status dyn_add_ball_joint(dyn_world* world, uint32_t first_body, uint32_t second_body, const float* anchor_a,
                                      const float* anchor_b, uint32_t* out_id);
/* ConstraintDescriptorRecords as dynamis-abi builds them (src/constraint.rs:109), appended in order
 * (all or nothing). On this path: DYN_CONSTRAINT_BALL with DISABLE_COLLISIONS, WARM_START and
 * HAS_BREAK; limits, swing cones and the other kinds return DYN_ERR_INVALID. */
DYN_API dyn_status dyn_add_constraints(dyn_world* world, const dyn_constraint_descriptor_record* records, uint32_t m,
                                       uint32_t* out_first_id);
DYN_API dyn_status dyn_constraint_count(const dyn_world* world, uint32_t* count);
/* The constraint runtime stream after the last step (accumulated impulses, reaction, broken), in
 * constraint order; m must equal dyn_constraint_count. */
DYN_API dyn_status dyn_read_constraints(dyn_world* world, dyn_constraint_runtime_record* out, uint32_t m);
/* Descriptors, body rows and initial runtime records of every constraint, for a checker. */
DYN_API dyn_status dyn_export_constraints(const dyn_world* world, dyn_constraint_descriptor_record* descs,
                                          dyn_constraint_rows_record* rows, dyn_constraint_runtime_record* runtime);
/* The joint solve order (crates/dynamis-world/src/schedule.rs:105-296): joint rows layer by layer,
 * (first row, count) per layer and (first layer, layer count) per component, in the planner's
 * component order. Any output may be NULL; sizes come back in *layer_count / *component_count. */
DYN_API dyn_status dyn_joint_plan(const dyn_world* world, uint32_t* rows, uint32_t* layers, uint32_t* components,
                                  uint32_t* layer_count, uint32_t* component_count);

/* No counterpart in the reference. The same stable LSD sort as dyn_radix_sort for callers that
 * cannot allocate device memory (an external pool that forbids out-of-band allocations, or a path
 * where cudaMalloc / cudaFree would synchronise the device): it needs no world and allocates
 * nothing. Its scratch is one file-scope device array sized for DYN_STATIC_SORT_MAX_KEYS keys
 * (about 4.2 MB, held by every GPU that loads the library until exit); larger n returns
 * DYN_ERR_CAPACITY. Keys and payload are device pointers, sorted in place on cuda_stream (NULL =
 * the legacy default stream); the call is asynchronous. All calls on a device share the array,
 * so calls that overlap on the GPU race and must be serialised by the caller. The first call on
 * a device (with that device current) looks up the array's address; make it before any stream
 * capture. */
#define DYN_STATIC_SORT_MAX_KEYS 262144u
DYN_API dyn_status dyn_radix_sort_static(uint32_t* major, uint32_t* minor, uint32_t* payload, uint32_t n,
                                         uint32_t major_digits, uint32_t minor_digits, void* cuda_stream);
/* No counterpart in the reference. The status word of the latest dyn_radix_sort_static call on the
 * current device, read after cuda_stream's work: *out = 0 and DYN_OK when every look-back wait
 * completed; otherwise the DYN_STATUS_* bits (DYN_STATUS_LOOKBACK_TIMEOUT: a wait ran out and the
 * output is not sorted) and DYN_ERR_DEVICE_STATUS. The next dyn_radix_sort_static call clears it.
 * Allocates nothing. */
DYN_API dyn_status dyn_radix_sort_static_status(void* cuda_stream, uint32_t* out);

/* Device status bits (dyn_device_status, dyn_radix_sort_static_status). */
#define DYN_STATUS_LOOKBACK_TIMEOUT 1u   /* a sort or scan look-back wait ran out of polls */
#define DYN_STATUS_ISLAND_HOOKS 2u
#define DYN_STATUS_ADJOINT_UNSUPPORTED 4u  /* a reversed step met a contact the adjoint does not cover */

/* Launch shapes of the step's kernels, no counterpart in the reference (its wgpu passes use fixed
 * workgroup sizes). None of them changes a result, only the time a step takes. grid_blocks_per_sm:
 * the blocks per SM a grid-stride launch is capped at (1-64, default 16); solve_threads: threads per
 * block of the contact blocks' kernels, the solve, its prepare, the warm start and the position
 * passes (64, 128 or 256, default 128); gjk_blocks_per_sm, epa_blocks_per_sm: blocks per SM of the
 * persistent GJK and EPA kernels (1-16, defaults 6 and 8). Takes effect at the next dyn_step;
 * refused while a tape records. */
typedef struct dyn_launch_config {
    uint32_t grid_blocks_per_sm;
    uint32_t solve_threads;
    uint32_t gjk_blocks_per_sm;
    uint32_t epa_blocks_per_sm;
} dyn_launch_config;
DYN_API dyn_status dyn_set_launch_config(dyn_world* world, const dyn_launch_config* config);
DYN_API dyn_status dyn_get_launch_config(const dyn_world* world, dyn_launch_config* out);
/* The autotuner, no counterpart in the reference: on the world as it stands, times `steps` steps of
 * dt for each candidate launch configuration (coordinate descent over the four fields, two rounds,
 * every trial from the same saved state), and keeps the fastest (also written to best, its device
 * time per step to best_ms; either may be NULL). Afterwards the world holds the state it had before
 * the call, counters included. Needs a world that has stepped (its device state exists), no tape
 * recording and no queued body edits. Synchronises the world's stream. */
DYN_API dyn_status dyn_autotune(dyn_world* world, float dt, uint32_t steps, dyn_launch_config* best, float* best_ms);

/* World::snapshot / World::restore (crates/dynamis-world/src/snapshot.rs:64-90). dyn_snapshot_take
 * waits for the queued steps and copies the world's simulated state on the device (body rows and
 * cold fields, the archived contacts the next step warm-starts from, the frozen contacts, the
 * joints' runtime, counters), with the queued body commands and the step clock. dyn_snapshot_restore
 * puts it back, after which the steps repeat the ones that followed the snapshot bit for bit; it
 * abandons observations. A snapshot is tied to its world and scene: after a spawn, a removal, a
 * constraint change or a contact-stream widening, restore returns DYN_ERR_INVALID. Both are refused
 * while a tape records. The caller frees a snapshot with dyn_snapshot_free. */
typedef struct dyn_snapshot dyn_snapshot;
DYN_API dyn_status dyn_snapshot_take(dyn_world* world, dyn_snapshot** out);
DYN_API dyn_status dyn_snapshot_restore(dyn_world* world, const dyn_snapshot* snapshot);
DYN_API dyn_status dyn_snapshot_free(dyn_snapshot* snapshot);

/* Solver guards, no counterpart in the reference (0, the default, is the reference's solver).
 * DYN_SOLVER_GUARD_ROW_MASS: the reference solves a contact's points together against manifold row
 * masses (solver_contact_block.wgsl:14-29, manifold_row_mass), and for some manifolds (a tilted box
 * landing on three points whose arms do not balance) that Jacobi iteration diverges: the impulses
 * grow at least twofold per iteration and the bodies leave at hundreds of metres a second. With the
 * guard, a block whose points' normalised coupling matrix D^-1/2 A D^-1/2 has an eigenvalue of 1.9
 * or more (the reference's iteration diverges from 2) solves each point against count x its own
 * mass instead; every other
 * block, and so every step where no block fails, is bit for bit the reference's. Takes effect at
 * the next dyn_step; refused while a tape records (the adjoint differentiates the reference's
 * solver), and dyn_tape_begin refuses a guarded world. */
#define DYN_SOLVER_GUARD_ROW_MASS 1u
DYN_API dyn_status dyn_set_solver_guard(dyn_world* world, uint32_t flags);

/* World::set_ccd (crates/dynamis-world/src/body.rs:496-501): declares or clears continuous collision
 * for one body (also settable at spawn, dyn_body_desc.ccd). Only a simulated (dynamic, not
 * kinematic) body may declare it (DYN_ERR_INVALID otherwise); a changed flag queues a wake of the
 * body for the next step, as the reference's install_body does (body.rs:284-290). While any body
 * declares it, every step sweeps the candidate pairs of those bodies over the step's motion and
 * moves each to its earliest impact (ccd_sweep.wgsl, ccd_apply.wgsl), after the substeps and
 * before sleep. Refused while a tape records; dyn_tape_begin refuses a world with a CCD body. */
DYN_API dyn_status dyn_set_ccd(dyn_world* world, uint32_t body_id, int32_t enabled);

/* Clears the world's sticky device status word (dyn_sync keeps reporting it until this call or a
 * new scene upload). Synchronises the world's stream. No counterpart in the reference, which has
 * no device status word. */
DYN_API dyn_status dyn_clear_device_status(dyn_world* world);

/* Test hook, no counterpart in the reference: the next dyn_radix_sort on `world` (world NULL: the
 * next dyn_radix_sort_static call) starts every digit pass's tile tickets at skipped_tiles (0 or 1;
 * with 1 the first tile never runs, so the look-back words the other tiles wait on are never
 * published) and gives each look-back wait at most spin_limit polls. Every wait then ends within
 * the limit with DYN_STATUS_LOOKBACK_TIMEOUT set and the output unsorted; every write stays inside
 * the caller's n keys. One call only; later sorts use the normal limit (2^22 polls). */
DYN_API dyn_status dyn_debug_sort_fault(dyn_world* world, uint32_t skipped_tiles, uint32_t spin_limit);

/* ---- differentiation: World::step_backward ----
 * The adjoint of World::step over the frozen active contact set of each step, replacing the
 * reference's differentiable rollout of its step (crates/dynamis-world/src/step.rs:34-39 run
 * forward, the solver passes of crates/dynamis-rigid/src/solver.rs:304-333 reversed). A step
 * differentiates from the state its substeps start from to the state it ends in: integration,
 * warm start, the Jacobi contact blocks, advance and position correction, with each step's contact
 * set (pairs, normals, anchors in the bodies' frames, active clamps) held as the narrowphase found
 * it and each contact point's depth moving with the bodies to first order. Parameters: every
 * body's inverse mass and the scale of its inverse inertia tensor, every collider's friction.
 *
 * dyn_tape_begin starts a recorded trajectory: it checkpoints the world and every
 * checkpoint_interval-th later dyn_step checkpoints again (body rows, archived contacts, counters).
 * dyn_step_backward reverses the last not yet reversed step: it restores the checkpoint of that
 * step's segment, steps the segment again with its snapshots taped (narrowphase included), and runs
 * the reverse graph. dyn_tape_end restores the state after the last recorded step and releases the
 * tape. Requirements (DYN_ERR_INVALID otherwise): sleeping off (config sleep_time = +inf), no
 * constraints, dynamic bodies with isotropic inverse inertia, while recording only body edits of
 * kind PATCH and no spawns or removals, one timestep for every recorded step. Contacts with soft
 * compliance, rolling or spin friction raise DYN_STATUS_ADJOINT_UNSUPPORTED (dyn_sync reports it).
 * The world's bodies hold replayed states between dyn_step_backward calls. */
typedef struct dyn_body_grad {
    float position[3];
    float _pad0;
    float orientation[4];      /* x, y, z, w */
    float velocity[3];
    float _pad1;
    float angular_velocity[3];
    float _pad2;
} dyn_body_grad;               /* 64 bytes: d loss / d one body row's state */

DYN_API dyn_status dyn_tape_begin(dyn_world* world, uint32_t checkpoint_interval);
DYN_API dyn_status dyn_tape_end(dyn_world* world);
DYN_API dyn_status dyn_tape_steps(const dyn_world* world, uint32_t* recorded, uint32_t* reversed);
/* World::step_backward: grad_in[row] = d loss / d (state after the step), n = body rows; writes
 * grad_out[row] = d loss / d (state its solve starts from, after the step's queued edits), and
 * adds the step's parameter gradients to the world's (dyn_param_grads). */
DYN_API dyn_status dyn_step_backward(dyn_world* world, const dyn_body_grad* grad_in, dyn_body_grad* grad_out, uint32_t n);
/* `steps` reversed steps in a row on the device (the state gradients stay in HBM between them;
 * a field a step's PATCH edit replaced passes no gradient to the step before it). */
DYN_API dyn_status dyn_backward(dyn_world* world, const dyn_body_grad* grad_in, dyn_body_grad* grad_out, uint32_t n,
                                uint32_t steps);
/* Parameter gradients accumulated since dyn_tape_begin: per body row d loss / d inverse mass and
 * d loss / d s at s = 1 for the inverse inertia tensor scaled by s (so for a mass m with inertia
 * proportional to it, d loss / d m = -(inverse_mass x g_inverse_mass + g_inertia_scale) / m); per
 * collider d loss / d friction. Any output may be NULL. */
DYN_API dyn_status dyn_param_grads(dyn_world* world, float* inverse_mass, float* inertia_scale, uint32_t n, float* friction,
                                   uint32_t k);
/* Sets body rows' inverse mass and inverse inertia tensor (6 per row: xx, xy, xz, yy, yz, zz; the
 * inertia is its inverse) and colliders' friction, on the host records and the device. No
 * counterpart in the reference (its bodies take mass at spawn); the parameters of a differentiable
 * rollout. Refused while a tape is recording. */
DYN_API dyn_status dyn_set_mass_properties(dyn_world* world, const float* inverse_mass, const float* inverse_inertia,
                                           uint32_t n);
DYN_API dyn_status dyn_set_friction(dyn_world* world, const float* friction, uint32_t k);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* DYNAMIS_CUDA_H */
