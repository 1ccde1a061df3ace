// layout.cuh - HBM layout of one world on the device.
//
// Bodies: one 128-byte BodyHot row per body holds every field the contact solver touches, so a
// solver thread pulls a body in four 32-byte sectors; colder per-body fields live in parallel
// arrays. Colliders and contacts are structure-of-arrays so warps read coalesced float4 columns.
// The host converts the byte-exact ABI records (include/dynamis_abi.h) to and from this layout.
#pragma once

#include <cstdint>

#include "dynamis_abi.h"

namespace dyn {

struct __align__(128) BodyHot {
    float4 pos;  // position.xyz, inverse_mass
    float4 rot;  // orientation (x, y, z, w)
    float4 vel;  // velocity.xyz, 0
    float4 ang;  // angular_velocity.xyz, 0
    float4 com;  // local centre of mass.xyz, 0
    float4 ii0;  // inverse inertia (xx, xy, xz, yy)
    float4 ii1;  // inverse inertia (yz, zz), 0, 0
    uint4 aux;   // sleeping, descriptor flags, contacts touching this body this step, 0
};
static_assert(sizeof(BodyHot) == 128, "BodyHot is one 128-byte row");

// Contacts in manifold-slot-major structure-of-arrays: point slot p of contact i is at [p * cap + i].
struct ContactSet {
    float4* normal;  // normal.xyz, friction
    uint4* rows;     // body row a, body row b, point_count | sensor << 8, events
    float4* mat;     // rolling_friction, spin_friction, relaxation, damping_ratio
    uint4* ids;      // collider a, collider b, first_body_id, second_body_id
    uint4* ids2;     // first_generation, second_generation, surface, triangle
    float4* extra;   // restitution, carried_normal, carried_tangent, 0
    float4* la;      // local_a.xyz, depth
    float4* lb;      // local_b.xyz, target speed
    float4* acc;     // accumulated normal, tangent 1, tangent 2, feature (bits)
    float4* pos;     // position.xyz, 0
};

// Pose-only terms of the contact blocks, rebuilt once per substep (point slot p of contact i at
// [p * cap + i], like ContactSet).
struct SolverRows {
    float4* arm_a;     // contact point - first body's world centre of mass, normal effective mass
    float4* arm_b;     // contact point - second body's world centre of mass, unsplit normal mass
    float4* masses;    // tangent-1 and tangent-2 effective masses, depth, target speed
    float4* tangent1;  // [cap] tangent 1, twist mass
    float4* tangent2;  // [cap] tangent 2, 0
};

// Control words (device-side counts the graph's kernels read instead of host values).
enum Ctl : uint32_t {
    CTL_ENTRIES = 0,
    CTL_PAIRS = 1,
    CTL_CONTACTS = 2,
    CTL_APPENDED = 3,  // contacts the narrowphase appended (stored ones: the first c_cap)
    CTL_LIVE = 4,
    CTL_SOLVER_ROWS = 5,
    CTL_ARCHIVED = 6,
    CTL_ROUNDS = 7,
    CTL_STATUS = 8,
    CTL_LIST0 = 10,  // narrowphase class lists (3 words)
    CTL_EPA = 13,    // penetrating convex pairs queued for EPA
    CTL_HITS = 14,   // convex pairs queued for the manifold
    CTL_CELL_OVERFLOW = 15,  // the cell table could not place a run: lookups fall back to searching
    CTL_GJK_NEXT = 16,       // next convex pair ticket of the GJK kernel
    CTL_GJK_PAIRS = 17,      // convex pairs past the centre-axis rejection
    CTL_PROBES = 18,         // separated convex pairs queued for the penetration probe
    CTL_EPA_NEXT = 19,       // next penetrating pair ticket of the EPA kernel
    CTL_STAGED = 20,         // contacts the narrowphase staged (every contact it found: at most one per pair)
    CTL_CCD_HITS = 21,       // sweep hits the continuous-collision pass recorded
    CTL_RESTING = 22,        // frozen contacts in the store the next step reads (kept across steps)
    CTL_REST_NEXT = 23,      // frozen contacts this step's commit wrote
    CTL_COUNT = 32
};

// The grid index in three sorted runs (grid_resting_*.wgsl, immovable_entries.wgsl): the entries of
// awake movable colliders, emitted and sorted every step; the immovable colliders' and the resting
// (movable, asleep) colliders' entries, kept sorted across steps and emitted again only when a
// member, its box or the grid resolution changed. Every collider owns the entry slots
// [8 * collider, 8 * collider + 8), so a kept run's entries stay where it left them; the step merges
// the three runs into one sorted list for the pair and cell kernels.
enum GridRun : uint32_t { RUN_AWAKE = 0, RUN_IMMOVABLE = 1, RUN_RESTING = 2, RUN_NONE = 3 };
// Words of the kept runs (`DeviceWorld::held`): outside the control words and counters, because a
// checkpoint restores those while the runs stay as the last step left them.
enum Held : uint32_t {
    HELD_STALE = 0,        // per step: bit r set when kept run r must be emitted again
    HELD_AWAKE = 1,        // entries of the awake run this step
    HELD_IMMOVABLE = 2,    // entries in the kept immovable run
    HELD_RESTING = 3,      // entries in the kept resting run
    HELD_BASE = 4,         // bits of the base cell size the kept runs were emitted at
    HELD_SORT_IMMOVABLE = 7,  // per step: entries the immovable run's sort covers (0 when it is kept)
    HELD_SORT_RESTING = 8,
    HELD_SCRATCH = 9,      // a scan total nothing reads
    HELD_LIST_KEPT = 10,   // per step: the merged list, cell table and run extents are the previous step's
    HELD_LIST_CLEAN = 11,  // the merged list holds no awake entry and only the kept runs as they stand
    HELD_COUNT = 16
};

// Where a taped step's kernels write the adjoint's snapshots (the tape of adjoint.cuh, slot *slot);
// every pointer is null outside taped steps. Layouts: relay [slot][4c]; vel [slot][K*I][2n]
// (velocities, then angular velocities, at each velocity iteration's start); acc [slot][K*I][4c]
// (accumulated impulses there); res, cnt [slot][K*P][n] (resolution at each position iteration's
// start, contributions that iteration counted), point p of contact i at p * c + i.
struct TapeWrites {
    const uint32_t* slot;
    uint32_t* relay;
    float4* vel;
    float4* acc;
    float4* res;
    uint32_t* cnt;
    uint32_t substeps, iterations, piterations;
    size_t n, c;
};

struct DeviceWorld {
    uint32_t n;   // body rows
    uint32_t nd;  // dynamic rows (rows [0, nd))
    uint32_t k;   // colliders
    uint32_t e_cap, p_cap, c_cap;
    uint32_t s_cap;  // the staging set's capacity (the pair stream's: a pair yields at most one contact)
    uint32_t n_cap;  // body rows the per-row buffers hold
    // bodies
    BodyHot* hot;
    float4* prev_pos;
    float4* prev_rot;
    float4* force;
    float4* torque;
    uint4* ident;  // body_id, generation, collision_group, collision_mask
    float* sleep_timer;
    float4* damp;    // linear_damping, angular_damping, gravity_scale, 0
    float2* thresh;  // sleep_velocity, sleep_angular_velocity
    float4* inert0;  // inertia (xx, xy, xz, yy)
    float2* inert1;  // inertia (yz, zz)
    uint32_t* activity;
    uint32_t* motion;
    uint32_t* wake_flags;
    uint32_t* row_of_id;
    uint32_t id_count;
    uint32_t* body_world;  // sub-world of each row (all 0 outside a batch)
    // continuous collision (ccd.cuh), per row: the bitwise complement of the earliest sweep hit's
    // time bits and of its (lower, higher collider) pair key, 0 when the row has none this step,
    // and that hit (normal + restitution, point + time)
    uint32_t* ccd_time;
    unsigned long long* ccd_key;
    float4* ccd_impact;  // [2n]
    // frozen contacts (freeze_contacts.wgsl, thaw_contacts.wgsl, island_link_resting.wgsl): the
    // contacts of body pairs that were both at rest when a step ended, kept across steps by body id
    // and generation. Two stores swap roles every step: a step reads rest_in (and its islands join
    // through it), and its commit writes the contacts that stay frozen, then the newly frozen ones,
    // into rest_out.
    uint4* rest_in;         // first_body_id, first_generation, second_body_id, second_generation
    uint2* rest_in_slots;   // collider a, collider b
    uint4* rest_out;
    uint2* rest_out_slots;
    uint32_t rest_cap;
    // colliders
    uint32_t* c_owner;
    uint4* c_kind;     // kind, flags, source, 0
    float4* c_offset;  // local_offset.xyz, radius
    float4* c_lrot;    // local_rotation
    float4* c_half;    // half_extents.xyz, half_height
    float4* c_mat;     // friction, restitution, rolling_friction, spin_friction
    float4* c_mat2;    // relaxation, damping_ratio, impact_force, 0
    uint2* c_filter;   // collision_group, collision_mask
    float4* c_scale;   // scale.xyz, 0
    const dyn_shape_source_record* sources;
    const float4* vertices;
    const uint4* hull_tris;        // every hull's outward triangles (vertex indices within its hull), hull by hull
    const uint2* hull_tri_range;   // [source]: first triangle, triangle count
    // broadphase
    float4* aabb;  // [2k]: min.xyz, max.xyz
    uint4* c_class;  // [k] per step: owner row, collision group, collision mask, kind | moves << 8 | unscaled << 9
    uint32_t* c_level;
    uint32_t* entry_count;
    uint32_t* entry_offset;
    uint32_t* ekey;
    uint32_t* eval;
    uint32_t* ekey_alt;
    uint32_t* eval_alt;
    float4* entries;  // [2e]: min.xyz + group bits, max.xyz + info bits; collider i's at slots [8i, 8i + 8)
    uint32_t* c_run;    // [k] per step: the GridRun a collider's entries belong to
    uint32_t* c_held;   // [k] the kept run whose entries the collider's slots hold (RUN_AWAKE: none)
    uint32_t* run_count;   // [3k] entries per collider and run this step emits (the scans' input)
    uint32_t* run_offset;  // [3k] their exclusive scan, the three runs' counts back to back
    uint32_t* run_key;     // [3e] the runs' cell keys, run r at [r * e_cap], sorted
    uint32_t* run_val;     // [3e] the runs' entry slots
    uint32_t* held;        // [HELD_COUNT]
    uint32_t* init_pos;    // [e] merged places of the entries that can start a same-cell pair: the awake run's, then the immovable run's
    uint2* cell_table;  // [1 << cell_bits]: (cell key, first sorted entry) per occupied cell
    uint2* erun;        // [e] per sorted entry: the first sorted entry of its cell run, the run's length
    uint32_t cell_bits;
    uint32_t* spill;  // host-mapped: [0] unused, [1] pairs attempted, [2] pairs refused (left by a refusing step),
                      // [3] contacts staged (the largest since the host looked)
    uint32_t* pmaj;  // candidate pairs in emission order (lower, higher collider slot)
    uint32_t* pmin;
    // narrowphase, its staging set (append order; point stride s_cap) and the compaction into pair order
    ContactSet tmp;
    uint32_t* cmaj;  // [s_cap] staged contacts' (lower, higher) collider slot, then sorted
    uint32_t* cmin;
    uint32_t* cval;  // staged contact of each sorted key
    uint32_t* cmaj_alt;
    uint32_t* cmin_alt;
    uint32_t* cval_alt;
    uint32_t* np_list;  // [4][p_cap] pair indices per narrowphase class, then the GJK's convex pairs
    uint32_t* epa_list;      // pair indices of penetrating convex pairs
    float4* epa_simplex;     // [4][slot]: the GJK simplex (w.xyz) EPA starts from
    uint32_t* probe_list;    // pair indices of separated convex pairs
    float4* probe_data;      // [6][slot]: their simplex, point count, distance, closest points, normal
    uint32_t* hit_list;      // pair indices of convex hits
    float4* hit_data;        // [2][slot]: point.xyz + distance, normal.xyz
    ContactSet cur;  // this step's contacts in sorted pair order
    ContactSet arc;  // last step's
    SolverRows srows;
    uint32_t* matched;
    // islands, live list, solver
    uint32_t* parents;
    uint32_t* istate;
    uint32_t* live;
    uint32_t* solver_rows;  // rows with a contact block, ascending
    uint32_t* row_flag;     // [n] 1 for a row with a contact block
    uint32_t* row_offset;   // [n] its place in solver_rows
    int32_t* vdelta;  // [8n]
    int32_t* pdelta;  // [8n]
    uint32_t* contributions;
    float4* resolution;
    // the position pass with its apply folded into the next iteration (worlds without joints)
    int4* pd3;              // [3][n_cap] rotating linear position deltas (x, y, z, 0)
    uint32_t* cnt3;         // [3][n_cap] rotating contribution counts
    float4* resolution_alt; // [n_cap] the resolution of odd iterations
    uint32_t* cowner;       // [c_cap] bit 0 / bit 1: the contact claimed its first / second row
    // constraints (ball joints) and their solve order
    uint32_t jcount;
    uint32_t jgroup_count;
    uint32_t jfilter_count;
    uint4* jmeta;       // kind, flags, first row, second row
    float4* janchor_a;  // anchor in the first body's frame, break force
    float4* janchor_b;  // anchor in the second body's frame, break torque
    dyn_constraint_runtime_record* jruntime;
    uint32_t* jrows;    // joints layer by layer
    uint2* jlayers;     // (first entry of jrows, count)
    uint2* jcomps;      // (first layer, layer count)
    uint4* jgroups;     // warp groups: first component, components, lanes each, deepest stack
    uint2* jfilter;     // sorted (lower row, higher row) of the joints that disable collisions
    uint32_t* jfilter_joint;
    // queued body edits of this step (runs of one row each; *edit_count runs)
    const dyn_body_edit_record* edits;
    const uint4* edit_runs;
    uint32_t* edit_count;
    // counters (reference slots) and control words
    uint32_t* counters;
    uint32_t* ctl;
    // a taped step (differentiation): where the step's kernels write the adjoint's snapshots
    TapeWrites tape;
    // DYN_SOLVER_GUARD_* bits (dyn_set_solver_guard); 0 is the reference's solver
    uint32_t solver_guard;
};

}  // namespace dyn
