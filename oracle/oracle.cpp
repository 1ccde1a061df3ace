// oracle.cpp - CPU restatement of one Dynamis rigid-body step (World::step), the parity checker.
//
// TEST INFRASTRUCTURE ONLY. tests/ load the shared library built from this file (ctypes) to check
// the CUDA product on identical inputs, and bench.py times it as the CPU baseline. The product
// package never includes, links or loads it.
//
// Pass order follows crates/dynamis-rigid/src/lib.rs:119-153 and the record() functions of
// apply_commands.rs:267-295, integrate.rs:90-107, emit_entries.rs:127-145,
// crates/dynamis-broadphase/src/passes.rs:145-160, narrowphase.rs:110-133, islands.rs:237-258,
// wake.rs, live.rs, solver.rs:76-95 and 304-333, commit.rs. Where the reference's output order
// depends on atomics (entry slots, pair emission, live list, solver rows) the oracle takes
// ascending order; parity is asserted on the order-independent results (sorted keys, sorted
// pairs, contacts, island ids, body states).
//
// Parity status: the reference (Rust + WGSL on wgpu) cannot run here and ships no numeric golden
// vectors for this path, so bit-level agreement with its own output is unpinned; this restatement
// is pinned against the known-answer behaviours of the reference's tests instead.
//
// Scope notes: the resting-region index (frozen grid entries and
// contacts of sleeping bodies) is replaced by re-emitting every movable collider each step with
// its awake bit, which yields the same candidate pairs for awake bodies; contact events are not
// published (only the CONTACT_ANNOUNCED flag that gates warm starting is kept).
//
// Threads: the loops the reference runs as data-parallel passes (AABBs, pair emission, the
// narrowphase, the contact solve and position blocks, integration, the applies) run on every host
// thread through OpenMP. Each shared write is an integer atomic (the fixed-point deltas, counters)
// or goes into per-block lists joined in index order, so every result, bit for bit, is the same for
// any thread count, including one.
#include <algorithm>
#include <cstring>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "dynamis_abi.h"
#include "oracle_geom.h"
#include "oracle_query.h"
#ifdef _OPENMP
#include <omp.h>
#endif

inline void atomic_add_u32(uint32_t* p, uint32_t v) { __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }
inline void atomic_max_u32(uint32_t* p, uint32_t v) {
    uint32_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
    while (cur < v && !__atomic_compare_exchange_n(p, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
}
// Runs fn(first, last, block) over [0, n) in blocks of `block` items on every thread.
template <typename F>
void parallel_blocks(size_t n, size_t block, F&& fn) {
    const long long blocks = (long long)((n + block - 1) / block);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long b = 0; b < blocks; ++b) {
        size_t first = (size_t)b * block;
        fn(first, std::min(n, first + block), (size_t)b);
    }
}

using namespace orc;

namespace {

// ---- grid: crates/dynamis-shader/shaders/grid_index.wgsl:28-287, core.wgsl:106-130 ----

constexpr float kGridScaleLimit = 1e12f;

struct I3 {
    int32_t x, y, z;
};
struct GridCells {
    I3 min, max;
};

inline float grid_extent_of(const Aabb& b) {
    return fmaxw(fmaxw(b.max.x - b.min.x, b.max.y - b.min.y), b.max.z - b.min.z);
}
inline float grid_scale_of(const Aabb& b) {
    float extent = grid_extent_of(b);
    if (extent <= 0.0f) return 0.0f;
    return clampw(1.0f / extent, 1.0f / kGridScaleLimit, kGridScaleLimit);
}
inline float grid_cell_size(uint32_t scale_bits, uint32_t extent_bits) {
    float scale = u2f(scale_bits);
    float extent = u2f(extent_bits);
    float finest = scale > 0.0f ? 1.0f / scale : kGridScaleLimit;
    return fmaxw(finest, extent * 9.31322574615478515625e-10f);  // exp2(-30)
}
inline int32_t f2i(float f) { return (int32_t)f; }  // values are already floored
inline I3 floor_div(V3 v, float cs) {
    return I3{f2i(std::floor(v.x / cs)), f2i(std::floor(v.y / cs)), f2i(std::floor(v.z / cs))};
}
inline GridCells grid_cells(const Aabb& box, float cs) { return GridCells{floor_div(box.min, cs), floor_div(box.max, cs)}; }
inline void grid_cell_span(const GridCells& c, uint32_t span[3]) {
    span[0] = (uint32_t)(c.max.x - c.min.x + 1);
    span[1] = (uint32_t)(c.max.y - c.min.y + 1);
    span[2] = (uint32_t)(c.max.z - c.min.z + 1);
}
inline uint32_t grid_cell_count(const GridCells& c) {
    uint32_t s[3];
    grid_cell_span(c, s);
    return s[0] * s[1] * s[2];
}
inline I3 grid_cell_at(const GridCells& c, uint32_t ordinal) {
    uint32_t s[3];
    grid_cell_span(c, s);
    uint32_t rows = s[1] * s[2];
    return I3{c.min.x + (int32_t)(ordinal / rows), c.min.y + (int32_t)((ordinal / s[2]) % s[1]),
              c.min.z + (int32_t)(ordinal % s[2])};
}
inline uint32_t grid_cell_offset(const GridCells& c, I3 coord) {
    return (uint32_t)(coord.x - c.min.x) | ((uint32_t)(coord.y - c.min.y) << 1) | ((uint32_t)(coord.z - c.min.z) << 2);
}
inline uint32_t cell_hash(I3 c) {
    uint32_t x = (uint32_t)c.x * 0x9E3779B9u;
    uint32_t y = (uint32_t)c.y * 0x85EBCA77u;
    uint32_t z = (uint32_t)c.z * 0xC2B2AE3Du;
    return (x ^ y ^ z ^ (x << 7) ^ (y >> 3) ^ (z << 11)) & DYN_CELL_HASH_MASK;
}
inline uint32_t cell_key(uint32_t level, I3 c) { return (level << DYN_LEVEL_KEY_SHIFT) | cell_hash(c); }
// Batched worlds (no counterpart in the reference): a row's sub-world is mixed into its cells'
// hash; sub-world 0 leaves the key unchanged.
inline uint32_t cell_key_in(uint32_t level, I3 c, uint32_t world) {
    return (level << DYN_LEVEL_KEY_SHIFT) | ((cell_hash(c) ^ (world * 0x2545F491u)) & DYN_CELL_HASH_MASK);
}
inline float level_cell_size(uint32_t level, float cs) { return cs * (float)(1u << level); }
inline uint32_t shape_levels(const Aabb& box, float base) {
    uint32_t level = 0;
    for (;;) {
        uint32_t s[3];
        grid_cell_span(grid_cells(box, level_cell_size(level, base)), s);
        uint32_t m = std::max(std::max(s[0], s[1]), s[2]);
        if (m <= DYN_MAX_CELLS_PER_AXIS || level >= DYN_GRID_LEVEL_LIMIT) break;
        level += 1;
    }
    return level;
}
inline bool i3eq(I3 a, I3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline bool aabb_overlaps(const Aabb& a, const Aabb& b) {
    return a.min.x <= b.max.x && a.min.y <= b.max.y && a.min.z <= b.max.z && b.min.x <= a.max.x
        && b.min.y <= a.max.y && b.min.z <= a.max.z;
}

// ---- LSD radix sort with 8-bit digits: crates/dynamis-sort/src/radix.rs:312-476 ----
// Stable; the minor word's digits go first, then the major word's (radix.rs:312-317).
void radix_sort_pairs(std::vector<uint32_t>& major, std::vector<uint32_t>& minor, std::vector<uint32_t>* payload,
                      uint32_t major_words, uint32_t minor_words) {
    size_t n = major.size();
    std::vector<uint32_t> tmp_major(n), tmp_minor(n), tmp_payload(payload ? n : 0);
    auto pass = [&](bool on_major, uint32_t digit) {
        uint32_t count[256] = {0};
        std::vector<uint32_t>& keys = on_major ? major : minor;
        for (size_t i = 0; i < n; ++i) count[(keys[i] >> (8 * digit)) & 255u] += 1;
        uint32_t offset[256];
        uint32_t run = 0;
        for (int d = 0; d < 256; ++d) {
            offset[d] = run;
            run += count[d];
        }
        for (size_t i = 0; i < n; ++i) {
            uint32_t d = (keys[i] >> (8 * digit)) & 255u;
            uint32_t dst = offset[d]++;
            tmp_major[dst] = major[i];
            tmp_minor[dst] = minor[i];
            if (payload) tmp_payload[dst] = (*payload)[i];
        }
        major.swap(tmp_major);
        minor.swap(tmp_minor);
        if (payload) payload->swap(tmp_payload);
    };
    for (uint32_t d = 0; d < minor_words; ++d) pass(false, d);
    for (uint32_t d = 0; d < major_words; ++d) pass(true, d);
}
// radix.rs:71-74: digits needed to hold values below n.
uint32_t key_words(uint32_t n) {
    uint32_t m = n > 0 ? n - 1 : 0;
    uint32_t bits = m == 0 ? 0 : 32 - (uint32_t)__builtin_clz(m);
    uint32_t words = (bits + 7) / 8;
    return words < 1 ? 1 : (words > 4 ? 4 : words);
}

struct Entry {
    Aabb box;
    uint32_t group;
    uint32_t info;
};

}  // namespace

struct OracleWorld {
    dyn_step_params params{};
    Shapes shapes;
    std::vector<dyn_shape_source_record> sources;
    std::vector<V4> vertices;
    std::vector<dyn_body_state_record> states;
    std::vector<dyn_body_descriptor_record> descs;
    std::vector<dyn_collider_record> colliders;
    std::vector<uint32_t> owners;
    std::vector<uint32_t> row_of_id;  // body_id -> row
    uint32_t pair_capacity = 0;
    uint32_t contact_capacity = 0;
    // per-step products kept for inspection
    uint32_t counters[DYN_COUNTER_DEVICE_COUNT] = {0};
    std::vector<Aabb> aabbs;
    std::vector<uint32_t> entry_keys, entry_order;
    std::vector<Entry> entries;
    std::vector<uint32_t> pair_major, pair_minor;
    std::vector<dyn_contact_record> contacts, archive;
    // the contacts as the substeps receive them (after the relay of accumulated impulses and the
    // target speeds), and for each of their points the archived point it was relayed from
    // (4 x held contact + held point, or -1): the frozen contact set of a differentiable step
    std::vector<dyn_contact_record> solve_contacts;
    std::vector<int32_t> relay_source;
    // the last step's branch decisions, for the differentiable step's reference: solve [substep]
    // [iteration][contact][point] (bit 0 normal impulse positive, 1/2 tangent-1 at its upper/lower
    // limit, 3 the tangent-2 limit passes a derivative (it is above 5 % of the friction limit), 4/5
    // tangent 2 at its upper/lower limit),
    // position [substep][iteration][contact][point] (bit 0 the point corrects), integrate
    // [substep][row] (bit 0 speed clamped, 1 spin clamped), targets [contact][point] (bit 0 from the
    // depth, 1 from restitution)
    std::vector<uint8_t> solve_flags, position_flags, integrate_flags, target_flags;
    uint32_t flag_substep = 0, flag_iteration = 0;
    // the last step's primal values where the differentiable step's reference evaluates its
    // derivatives: states at each substep's start [substep][row] (position, orientation, velocity,
    // angular velocity), velocities at
    // each velocity iteration's start [substep][iteration][row] (velocity, angular velocity),
    // accumulated impulses at each velocity iteration's start [substep][iteration][contact][point],
    // resolutions at each position iteration's start [substep][iteration][row]
    bool keep_snapshots = false;
    uint32_t solver_guard = 0;  // DYN_SOLVER_GUARD_* bits, the library's extension (0: the reference)
    std::vector<float> snap_pose, snap_vel, snap_acc, snap_res;
    std::vector<uint32_t> contact_matched;
    std::vector<uint32_t> island_parents, island_state;
    std::vector<uint32_t> wake_flags, body_activity, body_motion;
    std::vector<uint32_t> live;
    std::vector<uint32_t> block_counts, blocks, solver_rows;
    std::vector<float> target_speeds;
    std::vector<V3> resolution;
    std::vector<int32_t> velocity_deltas, position_deltas;
    std::vector<uint32_t> contributions;
    uint32_t solver_rounds = 0;
    // constraints (ball joints) and their solve order (schedule.rs:105-296)
    std::vector<dyn_constraint_descriptor_record> joint_descs;
    std::vector<dyn_constraint_rows_record> joint_rows;
    std::vector<dyn_constraint_runtime_record> joint_runtime;
    std::vector<uint32_t> plan_rows, plan_layers, plan_components;
    std::vector<uint32_t> body_world;  // sub-world of every row (empty: one world)
    // the kept grid runs (grid_resting_*.wgsl, immovable_entries.wgsl): the run whose entries each
    // collider's slots hold (0 none, 1 immovable, 2 resting), the box they were emitted with, and the
    // base cell size both kept runs were emitted at
    std::vector<uint32_t> held_run;
    std::vector<Aabb> held_box;
    uint32_t held_base = 0;
    // frozen contacts (freeze_contacts.wgsl): pairs of bodies both at rest when a step ended, by
    // body id and generation with their colliders, kept across steps in the order they were frozen
    struct Frozen {
        uint32_t first_id, first_generation, second_id, second_generation, a, b;
    };
    std::vector<Frozen> resting;
    // every hull's triangles (index triples over its vertices) and each source's (first, count)
    std::vector<uint32_t> hull_tris, hull_tri_ranges;
    // body commands queued for the next step: (row, edit), in command order
    std::vector<std::pair<uint32_t, dyn_body_edit_record>> edits;
    uint32_t world_of(uint32_t row) const { return body_world.empty() ? 0u : body_world[row]; }
};

namespace {

const uint32_t kPerStepCounters[] = {
    DYN_COUNTER_ENTRIES, DYN_COUNTER_RESTING_REBUILD, DYN_COUNTER_RESTING_SORT, DYN_COUNTER_IMMOVABLE_EMITTED,
    DYN_COUNTER_PAIRS, DYN_COUNTER_GRID_LEVELS, DYN_COUNTER_CONTACTS, DYN_COUNTER_JOINTS, DYN_COUNTER_EVENTS,
    DYN_COUNTER_REFUSED_PAIRS, DYN_COUNTER_REFUSED_EVENTS, DYN_COUNTER_ENTRY_FAULTS, DYN_COUNTER_REFUSED_RESTING,
    DYN_COUNTER_SLEPT, DYN_COUNTER_WOKE, DYN_COUNTER_ACTIVE, DYN_COUNTER_WOKE_DEFERRED, DYN_COUNTER_RESTING_GATHER,
    DYN_COUNTER_ISLANDS, DYN_COUNTER_ISLAND_FAULTS, DYN_COUNTER_SOLVE_LINEAR_RESIDUAL,
    DYN_COUNTER_SOLVE_ANGULAR_RESIDUAL, DYN_COUNTER_COARSE_ACTIVE, DYN_COUNTER_GRID_SCALE, DYN_COUNTER_GRID_EXTENT,
    DYN_COUNTER_BREAKS, DYN_COUNTER_PARTICLE_REACH, DYN_COUNTER_COARSE_NEIGHBOURS, DYN_COUNTER_LIVE,
    DYN_COUNTER_LIVE_FAULTS, DYN_COUNTER_ROW_FAULTS, DYN_COUNTER_SOFT_ACTIVE, DYN_COUNTER_SOFT_SLEPT,
    DYN_COUNTER_SOFT_WOKE, DYN_COUNTER_REFUSED_CONTACTS, DYN_COUNTER_IMPACTS, DYN_COUNTER_REFUSED_IMPACTS,
    DYN_COUNTER_SOFT_EVENTS, DYN_COUNTER_REFUSED_SOFT_EVENTS};

Body body_at(const OracleWorld& w, uint32_t row) { return load_body(w.states[row], w.descs[row]); }

// core.wgsl:229-255
bool body_is_active(const dyn_body_state_record& s, const dyn_body_descriptor_record& d) {
    return body_moves_d(d.inverse_mass, d.flags) && s.sleeping == 0u;
}
bool body_is_moving(const dyn_body_state_record& s, const dyn_body_descriptor_record& d, const dyn_step_params& p) {
    bool driven = body_moves_d(d.inverse_mass, d.flags) && !body_simulates_d(d.inverse_mass, d.flags);
    if (driven && (!veq(rd3(s.velocity), splat3(0.0f)) || !veq(rd3(s.angular_velocity), splat3(0.0f)))) return true;
    if (!body_simulates_d(d.inverse_mass, d.flags) || s.sleeping != 0u) return false;
    float sleep_v = (d.flags & DYN_OVERRIDE_SLEEP_LINEAR) ? d.sleep_velocity : p.sleep_velocity;
    float sleep_w = (d.flags & DYN_OVERRIDE_SLEEP_ANGULAR) ? d.sleep_angular_velocity : p.sleep_angular_velocity;
    return length(rd3(s.velocity)) > sleep_v || length(rd3(s.angular_velocity)) > sleep_w;
}

// body_edits.wgsl:11-21 (mark_disturbed)
void edit_disturbs(OracleWorld& w, uint32_t row, dyn_body_state_record& s, bool disturbed) {
    if (s.sleeping != 0u) {
        w.counters[DYN_COUNTER_WOKE] += 1;
        w.wake_flags[row] = 1u;
    } else if (disturbed) {
        w.wake_flags[row] = 1u;
    }
    s.sleeping = 0u;
    s.sleep_timer = 0.0f;
}

// body_edits.wgsl:35-103: every queued command of a row, in order. Rows run one after another
// here; on the device one thread takes each row's run (command.rs:157-176 groups them).
void apply_edits(OracleWorld& w) {
    for (const auto& [row, e] : w.edits) {
        if (row >= w.states.size()) continue;
        dyn_body_state_record& s = w.states[row];
        const dyn_body_descriptor_record& d = w.descs[row];
        const V3 ev = rd3(e.state.velocity), ep = rd3(e.state.position);
        if (e.kind == DYN_EDIT_PATCH) {
            if (e.mask & DYN_PATCH_POSITION) {
                wr3(s.position, ep);
                wr3(s.prev_position, ep);
            }
            if (e.mask & DYN_PATCH_ORIENTATION) {
                for (int k = 0; k < 4; ++k) s.orientation[k] = s.prev_orientation[k] = e.state.orientation[k];
            }
            if (e.mask & DYN_PATCH_VELOCITY) wr3(s.velocity, ev);
            if (e.mask & DYN_PATCH_ANGULAR_VELOCITY) wr3(s.angular_velocity, rd3(e.state.angular_velocity));
            bool teleport = (e.mask & (DYN_PATCH_POSITION | DYN_PATCH_ORIENTATION)) != 0u;
            edit_disturbs(w, row, s, teleport || !body_simulates_d(d.inverse_mass, d.flags));
        } else if (e.kind == DYN_EDIT_FORCE) {
            wr3(s.force, rd3(s.force) + rd3(e.state.force));
            edit_disturbs(w, row, s, false);
        } else if (e.kind == DYN_EDIT_FORCE_AT_POINT) {
            V3 f = rd3(e.state.force);
            wr3(s.force, rd3(s.force) + f);
            wr3(s.torque, rd3(s.torque) + cross(ep - body_com(load_body(s, d)), f));
            edit_disturbs(w, row, s, false);
        } else if (e.kind == DYN_EDIT_TORQUE) {
            wr3(s.torque, rd3(s.torque) + rd3(e.state.torque));
            edit_disturbs(w, row, s, false);
        } else if (e.kind == DYN_EDIT_IMPULSE) {
            wr3(s.velocity, rd3(s.velocity) + ev * d.inverse_mass);
            edit_disturbs(w, row, s, false);
        } else if (e.kind == DYN_EDIT_IMPULSE_AT_POINT) {  // apply_impulse_at, body_edits.wgsl:23-33
            wr3(s.velocity, rd3(s.velocity) + ev * d.inverse_mass);
            Body b = load_body(s, d);
            V3 lever = ep - body_com(b);
            wr3(s.angular_velocity, rd3(s.angular_velocity) + apply_inverse_inertia(b, cross(lever, ev)));
            edit_disturbs(w, row, s, false);
        } else if (e.kind == DYN_EDIT_ANGULAR_IMPULSE) {
            Body b = load_body(s, d);
            wr3(s.angular_velocity, rd3(s.angular_velocity) + apply_inverse_inertia(b, rd3(e.state.angular_velocity)));
            edit_disturbs(w, row, s, false);
        } else if (e.kind == DYN_EDIT_SLEEP) {
            if (s.sleeping == 0u) w.counters[DYN_COUNTER_SLEPT] += 1;
            // freeze_body, core.wgsl:218-227
            wr3(s.velocity, splat3(0.0f));
            wr3(s.angular_velocity, splat3(0.0f));
            wr3(s.force, splat3(0.0f));
            wr3(s.torque, splat3(0.0f));
            for (int k = 0; k < 3; ++k) s.prev_position[k] = s.position[k];
            for (int k = 0; k < 4; ++k) s.prev_orientation[k] = s.orientation[k];
            s.sleep_timer = 0.0f;
            s.sleeping = 1u;
            w.wake_flags[row] = 0u;
        } else if (e.kind == DYN_EDIT_WAKE) {
            if (s.sleeping != 0u) w.counters[DYN_COUNTER_WOKE] += 1;
            s.sleep_timer = 0.0f;
            s.sleeping = 0u;
            w.wake_flags[row] = 1u;
        }
    }
    w.edits.clear();
}

// apply_commands.rs:267-295: reset_counters.wgsl, clear_inputs.wgsl, body_edits.wgsl, activity.wgsl
void apply_commands(OracleWorld& w) {
    // joint_filter.wgsl: the jointed pairs filtered this step
    uint32_t jointed = 0;
    for (size_t j = 0; j < w.joint_descs.size(); ++j) {
        if (w.joint_runtime[j].broken == 0u && (w.joint_descs[j].flags & DYN_CONSTRAINT_DISABLE_COLLISIONS)) ++jointed;
    }
    for (uint32_t slot : kPerStepCounters) w.counters[slot] = 0;
    w.counters[DYN_COUNTER_JOINTS] = jointed;
    uint32_t n = (uint32_t)w.states.size();
    for (uint32_t i = 0; i < n; ++i) {
        wr3(w.states[i].force, splat3(0.0f));
        wr3(w.states[i].torque, splat3(0.0f));
    }
    apply_edits(w);
    w.body_activity.assign(n, 0);
    w.body_motion.assign(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
        bool awake = body_is_active(w.states[i], w.descs[i]);
        w.body_activity[i] = awake ? 1u : 0u;
        w.body_motion[i] = body_is_moving(w.states[i], w.descs[i], w.params) ? 1u : 0u;
        if (awake) w.counters[DYN_COUNTER_ACTIVE] = 1;
    }
}

// begin_step.wgsl:5-14 (dynamic rows); broadphase_aabb.wgsl:11-62 (colliders)
void prepare(OracleWorld& w) {
#pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < w.params.dynamic_count; ++i) {
        dyn_body_state_record& s = w.states[i];
        if (s.sleeping != 0u) continue;
        for (int k = 0; k < 3; ++k) s.prev_position[k] = s.position[k];
        for (int k = 0; k < 4; ++k) s.prev_orientation[k] = s.orientation[k];
    }
    uint32_t k = (uint32_t)w.colliders.size();
    w.aabbs.assign(k, Aabb{splat3(0.0f), splat3(0.0f)});
#pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < k; ++i) {
        uint32_t owner = w.owners[i];
        if (owner == DYN_NO_BODY) continue;
        const dyn_body_state_record& s = w.states[owner];
        const dyn_body_descriptor_record& d = w.descs[owner];
        const dyn_collider_record& c = w.colliders[i];
        WorldShape shape = world_collider(rd3(s.position), rd4(s.orientation), c);
        Aabb tight = world_aabb_of(w.shapes, shape);
        WorldShape upright = shape;
        upright.rotation = V4{0.0f, 0.0f, 0.0f, 1.0f};
        Aabb resolution = world_aabb_of(w.shapes, upright);
        atomic_max_u32(&w.counters[DYN_COUNTER_GRID_SCALE], f2u(grid_scale_of(resolution)));
        atomic_max_u32(&w.counters[DYN_COUNTER_GRID_EXTENT], f2u(fmaxw(grid_extent_of(resolution), 0.0f)));
        Aabb swept = tight;
        if (body_moves_d(d.inverse_mass, d.flags)) {
            V3 travel = vabs(rd3(s.velocity) * w.params.dt);
            float spin = length(rd3(s.angular_velocity) * w.params.dt);
            Body b = load_body(s, d);
            V3 center = rd3(s.position) + quat_rotate(rd4(s.orientation), rd3(c.local_offset));
            float radius = length((tight.max - tight.min) * 0.5f) + length(center - body_com(b));
            float reach_r = spin >= 3.141592653589793f ? 2.0f * radius : 2.0f * radius * osin(0.5f * spin);
            V3 reach = splat3(w.params.contact_margin + reach_r);
            swept.min = tight.min - travel - reach;
            swept.max = tight.max + travel + reach;
        }
        w.aabbs[i] = swept;
    }
}

float grid_base_cell(const OracleWorld& w) {
    return grid_cell_size(w.counters[DYN_COUNTER_GRID_SCALE], w.counters[DYN_COUNTER_GRID_EXTENT]);
}

// immovable_entries.wgsl:8-29, collider_entries.wgsl:9-35, collider_emit.wgsl:6-63, then the
// entry sort (broadphase/src/passes.rs:76-90: 4 digit passes over the cell key, payload = slot).
//
// The entries fall in three runs: awake movable colliders', emitted every step; immovable colliders'
// and resting (movable, asleep) colliders', which the library keeps sorted across steps and emits
// again only when a member joined or left, a member's box changed, or the grid resolution moved.
// The entry list is the same either way; what the runs change are the counters: ENTRIES and
// GRID_LEVELS count the awake run, RESTING_ENTRIES / RESTING_LEVELS and IMMOVABLE_ENTRIES /
// IMMOVABLE_LEVELS the kept runs, and IMMOVABLE_EMITTED, RESTING_REBUILD and RESTING_SORT what this
// step emitted again (grid_resting_gate.wgsl, grid_resting_commit.wgsl).
void emit_entries(OracleWorld& w) {
    float base = grid_base_cell(w);
    w.counters[DYN_COUNTER_IMMOVABLE_LEVELS] = 0;
    w.counters[DYN_COUNTER_IMMOVABLE_ENTRIES] = 0;
    w.counters[DYN_COUNTER_RESTING_LEVELS] = 0;
    w.counters[DYN_COUNTER_RESTING_ENTRIES] = 0;
    std::vector<uint32_t> keys, order;
    w.entries.clear();
    uint32_t k = (uint32_t)w.colliders.size();
    if (w.held_run.size() != k) {
        w.held_run.assign(k, 0u);
        w.held_box.assign(k, Aabb{});
    }
    constexpr uint32_t kAwake = 0, kImmovable = 1, kResting = 2, kNone = 3;
    std::vector<uint32_t> run_of(k, kNone);
    uint32_t stale = 0;
    auto bits_equal = [](const Aabb& a, const Aabb& b) { return std::memcmp(&a, &b, sizeof(Aabb)) == 0; };
    // slots in collider order (the reference takes them from an atomic counter, so any order is
    // one of its possible layouts; the sorted keys do not depend on it).
    {
        for (uint32_t i = 0; i < k; ++i) {
            uint32_t owner = w.owners[i];
            if (owner == DYN_NO_BODY) continue;
            const dyn_body_descriptor_record& d = w.descs[owner];
            bool moves = body_moves_d(d.inverse_mass, d.flags);
            bool awake = w.body_activity[owner] != 0u || w.wake_flags[owner] != 0u;
            const Aabb& box = w.aabbs[i];
            uint32_t level = shape_levels(box, base);
            const uint32_t run = !moves ? kImmovable : (awake ? kAwake : kResting);
            run_of[i] = run;
            uint32_t level_counter = run == kAwake ? DYN_COUNTER_GRID_LEVELS
                                     : run == kResting ? DYN_COUNTER_RESTING_LEVELS : DYN_COUNTER_IMMOVABLE_LEVELS;
            w.counters[level_counter] |= 1u << level;
            if (run != kAwake && !(w.held_run[i] == run && bits_equal(w.held_box[i], box))) stale |= 1u << run;
            GridCells cells = grid_cells(box, level_cell_size(level, base));
            uint32_t count = grid_cell_count(cells);
            uint32_t emitted = std::min(count, DYN_MAX_CELLS_PER_COLLIDER);
            if (count > emitted) w.counters[DYN_COUNTER_ENTRY_FAULTS] += count - emitted;
            if (level > 0u && awake) w.counters[DYN_COUNTER_COARSE_ACTIVE] += 1;
            for (uint32_t ordinal = 0; ordinal < emitted; ++ordinal) {
                I3 coord = grid_cell_at(cells, ordinal);
                uint32_t offset = grid_cell_offset(cells, coord);
                uint32_t info = i | (offset << DYN_ENTRY_CELL_SHIFT) | (DYN_ENTRY_KIND_COLLIDER << DYN_ENTRY_KIND_SHIFT);
                if (moves && awake) info |= DYN_ENTRY_AWAKE;
                if (moves) info |= DYN_ENTRY_MOBILE;
                if (offset == 0u) info |= DYN_ENTRY_PRIMARY;
                uint32_t slot = (uint32_t)w.entries.size();
                w.entries.push_back(Entry{box, owner, info});
                keys.push_back(cell_key_in(level, coord, w.world_of(owner)));
                order.push_back(slot);
                w.counters[run == kAwake ? DYN_COUNTER_ENTRIES
                           : run == kResting ? DYN_COUNTER_RESTING_ENTRIES : DYN_COUNTER_IMMOVABLE_ENTRIES] += 1;
            }
        }
    }
    // a collider that left a kept run makes it stale; so does a new grid resolution
    for (uint32_t i = 0; i < k; ++i) {
        if (w.held_run[i] != kAwake && w.held_run[i] != run_of[i]) stale |= 1u << w.held_run[i];
    }
    uint32_t base_bits;
    std::memcpy(&base_bits, &base, 4);
    if (base_bits != w.held_base) stale |= (1u << kImmovable) | (1u << kResting);
    w.held_base = base_bits;
    for (uint32_t i = 0; i < k; ++i) {
        const uint32_t run = run_of[i];
        if (run == kAwake || run == kNone) {
            w.held_run[i] = kAwake;
        } else if ((stale >> run) & 1u) {
            w.held_run[i] = run;
            w.held_box[i] = w.aabbs[i];
        }
    }
    const bool immovable = (stale >> kImmovable) & 1u, resting = (stale >> kResting) & 1u;
    w.counters[DYN_COUNTER_IMMOVABLE_EMITTED] = immovable ? w.counters[DYN_COUNTER_IMMOVABLE_ENTRIES] : 0u;
    w.counters[DYN_COUNTER_RESTING_REBUILD] = resting ? 1u : 0u;
    w.counters[DYN_COUNTER_RESTING_SORT] = resting ? w.counters[DYN_COUNTER_RESTING_ENTRIES] : 0u;
    std::vector<uint32_t> zero(keys.size(), 0);
    radix_sort_pairs(keys, zero, &order, 4, 0);
    w.entry_keys = keys;
    w.entry_order = order;
}

struct PairSink {
    const OracleWorld* w;
    std::vector<uint32_t> major, minor;
};

// pair_emit.wgsl:3-31
bool entry_awake(const OracleWorld& w, uint32_t node) {
    const Entry& e = w.entries[node];
    if ((e.info & DYN_ENTRY_MOBILE) == 0u) return w.wake_flags[e.group] != 0u;  // immovable region
    return (e.info & DYN_ENTRY_AWAKE) != 0u;
}
void emit_pair(PairSink& sink, uint32_t first, uint32_t second) {
    const Entry& a = sink.w->entries[first];
    const Entry& b = sink.w->entries[second];
    uint32_t ka = (a.info & DYN_ENTRY_KIND_MASK) >> DYN_ENTRY_KIND_SHIFT;
    uint32_t kb = (b.info & DYN_ENTRY_KIND_MASK) >> DYN_ENTRY_KIND_SHIFT;
    if (ka != DYN_ENTRY_KIND_COLLIDER || kb != DYN_ENTRY_KIND_COLLIDER) return;
    if (first == second || a.group == b.group) return;
    if ((a.info & DYN_ENTRY_MOBILE) == 0u && (b.info & DYN_ENTRY_MOBILE) == 0u) return;
    if (sink.w->world_of(a.group) != sink.w->world_of(b.group)) return;
    // the pair's slot (and the capacity cut) is taken when the blocks are joined in order
    uint32_t ia = a.info & DYN_ENTRY_INDEX_MASK;
    uint32_t ib = b.info & DYN_ENTRY_INDEX_MASK;
    sink.major.push_back(std::min(ia, ib));
    sink.minor.push_back(std::max(ia, ib));
}
I3 entry_cell(const Entry& e, float cs) {
    uint32_t bits = (e.info & DYN_ENTRY_CELL_MASK) >> DYN_ENTRY_CELL_SHIFT;
    I3 c = floor_div(e.box.min, cs);
    return I3{c.x + (int32_t)(bits & 1u), c.y + (int32_t)((bits >> 1) & 1u), c.z + (int32_t)((bits >> 2) & 1u)};
}
I3 grid_overlap_cell(const Aabb& a, const Aabb& b, float cs) { return floor_div(vmax(a.min, b.min), cs); }
void key_range(const OracleWorld& w, uint32_t key, uint32_t* first, uint32_t* last) {
    auto lo = std::lower_bound(w.entry_keys.begin(), w.entry_keys.end(), key);
    auto hi = std::upper_bound(w.entry_keys.begin(), w.entry_keys.end(), key);
    *first = (uint32_t)(lo - w.entry_keys.begin());
    *last = (uint32_t)(hi - w.entry_keys.begin());
}

// cell_pairs.wgsl:6-50 and level_links.wgsl:6-65, over one sorted entry array holding every
// region; then the pair sort (narrowphase.rs:110-126: collider_slot_words digits per word).
void broadphase(OracleWorld& w) {
    float grid = grid_base_cell(w);
    uint32_t occupied = w.counters[DYN_COUNTER_GRID_LEVELS] | w.counters[DYN_COUNTER_RESTING_LEVELS]
        | w.counters[DYN_COUNTER_IMMOVABLE_LEVELS];
    uint32_t live = (uint32_t)w.entry_keys.size();
    const size_t kBlock = 2048;
    const size_t blocks = (live + kBlock - 1) / kBlock;
    std::vector<PairSink> links(blocks, PairSink{&w, {}, {}}), cells(blocks, PairSink{&w, {}, {}});
    // level_links first, then cell_pairs (passes.rs record order); the pair set is what matters.
    parallel_blocks(live, kBlock, [&](size_t begin, size_t end, size_t b) {
        PairSink& sink = links[b];
        for (uint32_t index = (uint32_t)begin; index < (uint32_t)end; ++index) {
            uint32_t node = w.entry_order[index];
            const Entry& e = w.entries[node];
            if (((e.info & DYN_ENTRY_KIND_MASK) >> DYN_ENTRY_KIND_SHIFT) != DYN_ENTRY_KIND_COLLIDER) continue;
            if ((e.info & DYN_ENTRY_PRIMARY) == 0u) continue;
            bool awake = entry_awake(w, node);
            if (!awake && w.counters[DYN_COUNTER_COARSE_ACTIVE] == 0u) continue;
            uint32_t level = shape_levels(e.box, grid);
            uint32_t coarser = occupied & ~((1u << std::min(level + 1u, 31u)) - 1u);
            while (coarser != 0u) {
                uint32_t link = 31u - (uint32_t)__builtin_clz(coarser);
                coarser &= ~(1u << link);
                float cs = level_cell_size(link, grid);
                GridCells gc = grid_cells(e.box, cs);
                uint32_t count = grid_cell_count(gc);
                if ((long long)gc.max.x - gc.min.x > 3 || (long long)gc.max.y - gc.min.y > 3 ||
                    (long long)gc.max.z - gc.min.z > 3 || gc.max.x < gc.min.x || gc.max.y < gc.min.y ||
                    gc.max.z < gc.min.z) {
                    atomic_add_u32(&w.counters[DYN_COUNTER_ENTRY_FAULTS], 1u);  // non-finite box: same cut as the device
                    continue;
                }
                for (uint32_t ordinal = 0; ordinal < count; ++ordinal) {
                    I3 cell = grid_cell_at(gc, ordinal);
                    uint32_t first, last;
                    key_range(w, cell_key_in(link, cell, w.world_of(e.group)), &first, &last);
                    for (uint32_t entry = first; entry < last; ++entry) {
                        uint32_t other = w.entry_order[entry];
                        if (other == node) continue;
                        if (!awake && !entry_awake(w, other)) continue;
                        const Entry& o = w.entries[other];
                        if (!aabb_overlaps(e.box, o.box)) continue;
                        if (!i3eq(entry_cell(o, cs), cell)) continue;
                        if (!i3eq(grid_overlap_cell(e.box, o.box, cs), cell)) continue;
                        emit_pair(sink, node, other);
                    }
                }
            }
        }
    });
    parallel_blocks(live, kBlock, [&](size_t begin, size_t end, size_t b) {
        PairSink& sink = cells[b];
        for (uint32_t index = (uint32_t)begin; index < (uint32_t)end; ++index) {
            uint32_t node = w.entry_order[index];
            const Entry& e = w.entries[node];
            if (((e.info & DYN_ENTRY_KIND_MASK) >> DYN_ENTRY_KIND_SHIFT) != DYN_ENTRY_KIND_COLLIDER) continue;
            if (!entry_awake(w, node)) continue;
            uint32_t level = shape_levels(e.box, grid);
            float cs = level_cell_size(level, grid);
            I3 cell = entry_cell(e, cs);
            uint32_t first, last;
            key_range(w, cell_key_in(level, cell, w.world_of(e.group)), &first, &last);
            for (uint32_t entry = first; entry < last; ++entry) {
                if (entry == index) continue;
                uint32_t other = w.entry_order[entry];
                if (entry_awake(w, other) && entry < index) continue;
                const Entry& o = w.entries[other];
                if (!aabb_overlaps(e.box, o.box)) continue;
                if (!i3eq(entry_cell(o, cs), cell)) continue;
                if (!i3eq(grid_overlap_cell(e.box, o.box, cs), cell)) continue;
                emit_pair(sink, node, other);
            }
        }
    });
    // pair_emit.wgsl's slot counter: pairs beyond the capacity are refused, in emission order
    std::vector<uint32_t> major, minor;
    uint64_t emitted = 0;
    for (const std::vector<PairSink>* part : {&links, &cells}) {
        for (const PairSink& sink : *part) {
            for (size_t i = 0; i < sink.major.size(); ++i, ++emitted) {
                if (emitted >= w.pair_capacity) continue;
                major.push_back(sink.major[i]);
                minor.push_back(sink.minor[i]);
            }
        }
    }
    w.counters[DYN_COUNTER_PAIRS] = (uint32_t)emitted;
    w.counters[DYN_COUNTER_REFUSED_PAIRS] = (uint32_t)(emitted - major.size());
    links.clear();
    cells.clear();
    uint32_t words = key_words(std::max<uint32_t>((uint32_t)w.colliders.size(), 1u));
    radix_sort_pairs(major, minor, nullptr, words, words);
    w.pair_major = std::move(major);
    w.pair_minor = std::move(minor);
}

// narrowphase.wgsl:518-685 for one pair; false when the pair answers no contact.
// joint_filter.wgsl:9-24 then joined_pairs.wgsl: an unbroken joint with collisions disabled between
// the two rows. The reference rebuilds the sorted list every step; a scan of the joints is the same test.
bool joined_by_joint(const OracleWorld& w, uint32_t first_row, uint32_t second_row) {
    uint32_t a = std::min(first_row, second_row), b = std::max(first_row, second_row);
    for (size_t j = 0; j < w.joint_descs.size(); ++j) {
        if (w.joint_runtime[j].broken != 0u) continue;
        if ((w.joint_descs[j].flags & DYN_CONSTRAINT_DISABLE_COLLISIONS) == 0u) continue;
        const dyn_constraint_rows_record& r = w.joint_rows[j];
        if (std::min(r.first_row, r.second_row) == a && std::max(r.first_row, r.second_row) == b) return true;
    }
    return false;
}

bool narrowphase_pair(const OracleWorld& w, uint32_t first_slot, uint32_t second_slot, dyn_contact_record* out) {
    uint32_t fb = w.owners[first_slot];
    uint32_t sb = w.owners[second_slot];
    if (fb == DYN_NO_BODY || sb == DYN_NO_BODY || fb == sb) return false;
    Body first = body_at(w, fb);
    Body second = body_at(w, sb);
    if (!body_moves(first) && !body_moves(second)) return false;
    const dyn_collider_record& fc = w.colliders[first_slot];
    const dyn_collider_record& sc = w.colliders[second_slot];
    if (fc.kind == DYN_SHAPE_NONE || sc.kind == DYN_SHAPE_NONE) return false;
    uint32_t fg = fc.collision_group != DYN_NO_COLLISION_FILTER ? fc.collision_group : first.group;
    uint32_t fm = fc.collision_mask != DYN_NO_COLLISION_FILTER ? fc.collision_mask : first.mask;
    uint32_t sg = sc.collision_group != DYN_NO_COLLISION_FILTER ? sc.collision_group : second.group;
    uint32_t sm = sc.collision_mask != DYN_NO_COLLISION_FILTER ? sc.collision_mask : second.mask;
    if (!((fg & sm) != 0u && (sg & fm) != 0u)) return false;
    if (joined_by_joint(w, fb, sb)) return false;
    bool sensor = (fc.flags & DYN_COLLIDER_SENSOR) != 0u || (sc.flags & DYN_COLLIDER_SENSOR) != 0u;
    bool fw = shape_world_geometry(fc.kind);
    bool sw = shape_world_geometry(sc.kind);
    if (fw && sw) return false;
    float margin = w.params.contact_margin;
    if (body_has_ccd(first) || body_has_ccd(second)) {
        margin = w.params.contact_margin + length(second.velocity - first.velocity) * w.params.dt;
    }
    Manifold m;
    bool generated = false;
    const Shapes& sh = w.shapes;
    if (fw) {
        if (fc.kind != DYN_SHAPE_PLANE) return false;  // meshes / heightfields not restated
        WorldShape scene = world_collider(first.position, first.orientation, fc);
        WorldShape ws = world_collider(second.position, second.orientation, sc);
        m = plane_convex(sh, scene, ws, margin);
        generated = m.point_count > 0u;
    } else if (sw) {
        if (sc.kind != DYN_SHAPE_PLANE) return false;
        WorldShape scene = world_collider(second.position, second.orientation, sc);
        WorldShape wf = world_collider(first.position, first.orientation, fc);
        m = plane_convex(sh, scene, wf, margin);
        m.normal = -m.normal;
        mirror_features(&m);
        generated = m.point_count > 0u;
    } else if (scaled_shape(fc) || scaled_shape(sc) || !shape_analytic(fc.kind) || !shape_analytic(sc.kind)) {
        WorldShape wf = world_collider(first.position, first.orientation, fc);
        WorldShape ws = world_collider(second.position, second.orientation, sc);
        ShapeHit hit = convex_hit(sh, wf, ws);
        if (hit.distance <= margin) {
            manifold_emit(&m, hit.normal);
            generated = true;
            if (!convex_pair_manifold(sh, wf, ws, hit.normal, &m)) manifold_from_hit(&m, hit, margin);
        }
    } else {
        uint32_t a = fc.kind, b = sc.kind;
        if (a == DYN_SHAPE_SPHERE && b == DYN_SHAPE_SPHERE) {
            m = sphere_sphere(first, fc, second, sc, margin);
        } else if (a == DYN_SHAPE_SPHERE && b == DYN_SHAPE_CUBOID) {
            m = sphere_box(first, fc, second, sc, margin);
        } else if (a == DYN_SHAPE_SPHERE && b == DYN_SHAPE_CAPSULE) {
            m = sphere_capsule(first, fc, second, sc, margin);
        } else if (a == DYN_SHAPE_CUBOID && b == DYN_SHAPE_SPHERE) {
            m = sphere_box(second, sc, first, fc, margin);
            m.normal = -m.normal;
        } else if (a == DYN_SHAPE_CUBOID && b == DYN_SHAPE_CUBOID) {
            m = box_box_sat(first, fc, second, sc, margin);
        } else if (a == DYN_SHAPE_CAPSULE && b == DYN_SHAPE_SPHERE) {
            m = sphere_capsule(second, sc, first, fc, margin);
            m.normal = -m.normal;
        } else if (a == DYN_SHAPE_CAPSULE && b == DYN_SHAPE_CAPSULE) {
            m = capsule_capsule(first, fc, second, sc, margin);
        } else {
            WorldShape wf = world_collider(first.position, first.orientation, fc);
            WorldShape ws = world_collider(second.position, second.orientation, sc);
            ShapeHit hit = convex_hit(sh, wf, ws);
            if (hit.distance <= margin) {
                manifold_emit(&m, hit.normal);
                if (!convex_pair_manifold(sh, wf, ws, hit.normal, &m)) manifold_from_hit(&m, hit, margin);
            }
        }
        generated = true;
    }
    if (!generated || m.point_count == 0u) return false;
    dyn_contact_record c;
    std::memset(&c, 0, sizeof(c));
    c.a = first_slot;
    c.b = second_slot;
    c.point_count = m.point_count;
    c.sensor = sensor ? 1u : 0u;
    c.first_body_id = first.body_id;
    c.second_body_id = second.body_id;
    c.first_generation = first.generation;
    c.second_generation = second.generation;
    wr3(c.normal, m.normal);
    c.triangle = m.triangle;
    c.surface = DYN_NO_SURFACE;
    c.friction = material_combine(fc.friction, sc.friction, w.params.friction_combine);
    c.restitution = material_combine(fc.restitution, sc.restitution, w.params.restitution_combine);
    c.rolling_friction = fmaxw(fc.rolling_friction, sc.rolling_friction);
    c.spin_friction = fmaxw(fc.spin_friction, sc.spin_friction);
    c.relaxation = fc.relaxation + sc.relaxation;
    c.damping_ratio = fmaxw(fc.damping_ratio, sc.damping_ratio);
    c.events = (fc.flags & sc.flags) & (DYN_EVENT_MODE_BEGIN_END | DYN_EVENT_MODE_PERSIST);
    for (uint32_t i = 0; i < m.point_count; ++i) {
        dyn_manifold_point_record& p = c.points[i];
        V3 point = m.points[i].position;
        wr3(p.position, point);
        p.depth = m.points[i].depth;
        p.feature = m.points[i].feature;
        wr3(p.local_a, quat_rotate(quat_conjugate(first.orientation), point - first.position));
        wr3(p.local_b, quat_rotate(quat_conjugate(second.orientation), point - second.position));
    }
    *out = c;
    return true;
}

// narrowphase pass + compact_scan/offsets/scatter.wgsl: contacts in pair order.
void narrowphase(OracleWorld& w) {
    w.contacts.clear();
    const size_t p = w.pair_major.size();
    // pairs in blocks on every thread; the blocks' contacts are joined in pair order
    const size_t kBlock = 1024, kSpan = 64 * kBlock;
    std::vector<std::vector<dyn_contact_record>> found;
    for (size_t span = 0; span < p; span += kSpan) {
        const size_t n = std::min(kSpan, p - span);
        found.assign((n + kBlock - 1) / kBlock, {});
        parallel_blocks(n, kBlock, [&](size_t begin, size_t end, size_t b) {
            for (size_t i = span + begin; i < span + end; ++i) {
                dyn_contact_record c;
                if (!narrowphase_pair(w, w.pair_major[i], w.pair_minor[i], &c)) continue;
                c.carried_normal = 0.0f;
                c.carried_tangent = 0.0f;
                found[b].push_back(c);
            }
        });
        for (const std::vector<dyn_contact_record>& block : found) {
            for (const dyn_contact_record& c : block) {
                if (w.contacts.size() >= w.contact_capacity) {
                    w.counters[DYN_COUNTER_REFUSED_CONTACTS] += 1;
                    continue;
                }
                w.contacts.push_back(c);
            }
        }
    }
    w.counters[DYN_COUNTER_CONTACTS] = (uint32_t)w.contacts.size();
    w.contact_matched.assign(w.contacts.size(), 0);
}

// identity.wgsl:8-118
bool contact_touches(const dyn_contact_record& c, float threshold) {
    for (uint32_t i = 0; i < c.point_count; ++i) {
        if (c.points[i].depth >= -threshold) return true;
    }
    return false;
}
bool contact_same_pair(const dyn_contact_record& h, const dyn_contact_record& c) {
    bool same = h.first_body_id == c.first_body_id && h.first_generation == c.first_generation
        && h.second_body_id == c.second_body_id && h.second_generation == c.second_generation && h.a == c.a
        && h.b == c.b;
    bool flipped = h.first_body_id == c.second_body_id && h.first_generation == c.second_generation
        && h.second_body_id == c.first_body_id && h.second_generation == c.first_generation && h.a == c.b
        && h.b == c.a;
    return same || flipped;
}
float contact_normal_impulse(const dyn_contact_record& c) {
    float total = 0.0f;
    for (uint32_t i = 0; i < c.point_count; ++i) total = total + fmaxw(c.points[i].accumulated_normal, 0.0f);
    return total;
}
float contact_tangent_impulse(const dyn_contact_record& c) {
    float total = 0.0f;
    for (uint32_t i = 0; i < c.point_count; ++i) {
        const dyn_manifold_point_record& p = c.points[i];
        total = total + std::sqrt(p.accumulated_tangent_1 * p.accumulated_tangent_1
                                  + p.accumulated_tangent_2 * p.accumulated_tangent_2);
    }
    return total;
}
dyn_contact_record contact_relay_impulses(const dyn_contact_record& current, const dyn_contact_record& held,
                                          int32_t* source = nullptr, int32_t held_index = 0) {
    dyn_contact_record relayed = current;
    bool taken[4] = {false, false, false, false};
    for (uint32_t pi = 0; pi < current.point_count; ++pi) {
        const dyn_manifold_point_record& point = relayed.points[pi];
        uint32_t picked = DYN_NO_SLOT;
        float picked_distance = 0.0f;
        for (uint32_t hi = 0; hi < held.point_count; ++hi) {
            if (taken[hi]) continue;
            const dyn_manifold_point_record& hp = held.points[hi];
            if (!(hp.feature == point.feature || hp.feature == feature_mirror(point.feature))) continue;
            float distance = length(rd3(hp.local_a) - rd3(point.local_a)) + length(rd3(hp.local_b) - rd3(point.local_b));
            if (picked == DYN_NO_SLOT || distance < picked_distance) {
                picked = hi;
                picked_distance = distance;
            }
        }
        if (picked == DYN_NO_SLOT) continue;
        taken[picked] = true;
        if (source) source[pi] = 4 * held_index + (int32_t)picked;
        relayed.points[pi].accumulated_normal = held.points[picked].accumulated_normal;
        relayed.points[pi].accumulated_tangent_1 = held.points[picked].accumulated_tangent_1;
        relayed.points[pi].accumulated_tangent_2 = held.points[picked].accumulated_tangent_2;
    }
    return relayed;
}
uint32_t resolve_row(const OracleWorld& w, uint32_t id, uint32_t generation) {
    if (id >= w.row_of_id.size()) return DYN_NO_BODY;
    uint32_t row = w.row_of_id[id];
    if (row == DYN_NO_BODY || w.states[row].generation != generation) return DYN_NO_BODY;
    return row;
}

// contact_relay.wgsl:34-71 and contact_begin.wgsl:41-71 (event publication left out)
void relay_contacts(OracleWorld& w) {
    uint32_t count = (uint32_t)w.contacts.size();
    w.relay_source.assign(4 * (size_t)count, -1);
    for (size_t held_index = 0; held_index < w.archive.size(); ++held_index) {
        const dyn_contact_record& held = w.archive[held_index];
        uint32_t fr = resolve_row(w, held.first_body_id, held.first_generation);
        uint32_t sr = resolve_row(w, held.second_body_id, held.second_generation);
        if (fr == DYN_NO_BODY || sr == DYN_NO_BODY) continue;
        uint32_t lo = 0, hi = count;
        while (lo < hi) {
            uint32_t mid = (lo + hi) / 2;
            const dyn_contact_record& cand = w.contacts[mid];
            if (cand.a < held.a || (cand.a == held.a && cand.b < held.b)) {
                lo = mid + 1;
            } else {
                hi = mid;
            }
        }
        if (!(lo < count && w.contacts[lo].a == held.a && w.contacts[lo].b == held.b)) continue;
        dyn_contact_record current = w.contacts[lo];
        if (!contact_same_pair(held, current)) continue;
        if ((held.events & DYN_CONTACT_ANNOUNCED) == 0u) continue;
        w.contact_matched[lo] = 1;
        dyn_contact_record relayed = contact_relay_impulses(current, held, &w.relay_source[4 * (size_t)lo], (int32_t)held_index);
        relayed.carried_normal = contact_normal_impulse(relayed);
        relayed.carried_tangent = contact_tangent_impulse(relayed);
        relayed.events |= DYN_CONTACT_ANNOUNCED;
        w.contacts[lo] = relayed;
    }
    for (uint32_t i = 0; i < count; ++i) {
        if (w.contact_matched[i] != 0u) continue;
        if (contact_touches(w.contacts[i], w.params.slop)) w.contacts[i].events |= DYN_CONTACT_ANNOUNCED;
    }
}

// island_link.wgsl:1-45
uint32_t island_find(const OracleWorld& w, uint32_t node) {
    uint32_t current = node;
    uint32_t parent = w.island_parents[current];
    while (parent != current) {
        current = parent;
        parent = w.island_parents[current];
    }
    return current;
}
void island_couple(OracleWorld& w, uint32_t first, uint32_t second) {
    uint32_t dc = w.params.dynamic_count;
    // carry_static_wake(first, second) then carry_static_wake(second, first)
    if (second >= dc && w.wake_flags[second] != 0u) w.wake_flags[first] |= 1u;
    if (first >= dc && w.wake_flags[first] != 0u) w.wake_flags[second] |= 1u;
    if (first >= dc || second >= dc || first == second) return;
    uint32_t a = island_find(w, first);
    uint32_t b = island_find(w, second);
    if (a == b) return;
    uint32_t lower = std::min(a, b), higher = std::max(a, b);
    w.island_parents[higher] = lower;
}

// islands.rs:237-258 BuildIslands.record
void build_islands(OracleWorld& w) {
    relay_contacts(w);
    uint32_t dc = w.params.dynamic_count;
    w.island_parents.resize(dc);
    w.island_state.assign(dc, 0);
    for (uint32_t i = 0; i < dc; ++i) w.island_parents[i] = i;
    for (const dyn_contact_record& c : w.contacts) {
        if (c.point_count == 0u || c.sensor == 1u || !contact_touches(c, w.params.slop)) continue;
        island_couple(w, w.owners[c.a], w.owners[c.b]);
    }
    // island_link_constraints.wgsl
    for (size_t j = 0; j < w.joint_descs.size(); ++j) {
        if (w.joint_runtime[j].broken != 0u) continue;
        island_couple(w, w.joint_rows[j].first_row, w.joint_rows[j].second_row);
    }
    // island_link_resting.wgsl:10-21: the frozen contacts keep their sleeping bodies in one island
    for (const OracleWorld::Frozen& f : w.resting) {
        uint32_t first = resolve_row(w, f.first_id, f.first_generation);
        uint32_t second = resolve_row(w, f.second_id, f.second_generation);
        if (first == DYN_NO_BODY || second == DYN_NO_BODY) continue;
        island_couple(w, first, second);
    }
    uint32_t rounds = 32 - (uint32_t)__builtin_clz(std::max(dc, 2u));  // ilog2(max(N,2)) + 1
    for (uint32_t r = 0; r < rounds; ++r) {
        std::vector<uint32_t> next(dc);
        for (uint32_t i = 0; i < dc; ++i) {
            uint32_t parent = w.island_parents[i];
            next[i] = std::min(parent, w.island_parents[parent]);
        }
        w.island_parents.swap(next);
    }
    for (uint32_t i = 0; i < dc; ++i) {
        if (w.wake_flags[i] == 0u && w.body_motion[i] == 0u) continue;
        uint32_t root = w.island_parents[i];
        w.island_state[root] = std::max(w.island_state[root], DYN_ISLAND_WAKE);
    }
    for (uint32_t i = 0; i < dc; ++i) {
        if (w.island_parents[i] == i) w.counters[DYN_COUNTER_ISLANDS] += 1;
    }
}

// island_wake.wgsl:10-22 and live.wgsl:8-18
void wake_and_live(OracleWorld& w) {
    uint32_t dc = w.params.dynamic_count;
    for (uint32_t i = 0; i < dc; ++i) {
        uint32_t root = w.island_parents[i];
        dyn_body_state_record& s = w.states[i];
        if (s.sleeping != 0u && (w.island_state[root] & DYN_ISLAND_WAKE) != 0u) {
            w.counters[DYN_COUNTER_WOKE] += 1;
            w.counters[DYN_COUNTER_WOKE_DEFERRED] += 1;
            s.sleeping = 0;
            s.sleep_timer = 0.0f;
        }
        w.wake_flags[i] = 0;
    }
    w.live.clear();
    for (uint32_t i = 0; i < dc; ++i) {
        if (body_is_active(w.states[i], w.descs[i])) w.live.push_back(i);
    }
    w.counters[DYN_COUNTER_LIVE] = (uint32_t)w.live.size();
}

// core.wgsl:6-12
inline int32_t solver_word(float value, float scale) {
    return (int32_t)clampw(value * scale, -2.0e9f, 2.0e9f);
}
inline float solver_value(int32_t word, float scale) { return (float)word / scale; }

Body body_split(Body b, float scale) {
    b.inverse_mass = b.inverse_mass * scale;
    for (int i = 0; i < 6; ++i) b.inverse_inertia[i] = b.inverse_inertia[i] * scale;
    return b;
}
inline bool contact_block_resolves(const dyn_contact_record& c) { return c.point_count > 0u && c.sensor == 0u; }

// solver_reset.wgsl, solver_total.wgsl, solver_blocks.wgsl:24-48
void solver_prepare(OracleWorld& w) {
    uint32_t n = (uint32_t)w.states.size();
    uint32_t c = (uint32_t)w.contacts.size();
    w.block_counts.assign(n, 0);
    w.resolution.assign(n, splat3(0.0f));
    w.counters[DYN_COUNTER_BLOCKS] = c;
    w.counters[DYN_COUNTER_SOLVER_ROWS] = 0;
    w.blocks.assign(2 * (size_t)c, 0);
    w.target_speeds.assign(4 * (size_t)c, 0.0f);
    w.target_flags.assign(4 * (size_t)c, 0u);
    {
        const dyn_step_params& p = w.params;
        w.solve_flags.assign((size_t)p.substeps * p.solve_iterations * 4 * c, 0u);
        w.position_flags.assign((size_t)p.substeps * p.position_iterations * 4 * c, 0u);
        w.integrate_flags.assign((size_t)p.substeps * n, 0u);
    }
    w.solver_rows.clear();
    w.velocity_deltas.assign(8 * (size_t)n, 0);
    w.position_deltas.assign(8 * (size_t)n, 0);
    w.contributions.assign(n, 0);
    for (uint32_t index = 0; index < c; ++index) {
        const dyn_contact_record& contact = w.contacts[index];
        uint32_t fb = w.owners[contact.a];
        uint32_t sb = w.owners[contact.b];
        w.blocks[2 * index] = fb;
        w.blocks[2 * index + 1] = sb;
        if (!contact_block_resolves(contact)) continue;
        Body first = body_at(w, fb);
        Body second = body_at(w, sb);
        for (uint32_t pi = 0; pi < contact.point_count; ++pi) {
            V3 position = rd3(contact.points[pi].position);
            float speed = dot(relative_velocity(first, second, position, position), rd3(contact.normal));
            float target = 0.0f;
            if (contact.points[pi].depth < 0.0f) {
                target = contact.points[pi].depth / w.params.dt;
                w.target_flags[4 * (size_t)index + pi] = 1u;
            } else if (speed < -w.params.restitution_threshold) {
                target = -speed * contact.restitution;
                w.target_flags[4 * (size_t)index + pi] = 2u;
            }
            w.target_speeds[4 * (size_t)index + pi] = target;
        }
        for (uint32_t row : {fb, sb}) {
            if (w.block_counts[row]++ == 0u) {
                w.solver_rows.push_back(row);
                w.counters[DYN_COUNTER_SOLVER_ROWS] += 1;
            }
        }
    }
}

void accumulate(std::vector<int32_t>& deltas, uint32_t row, V3 linear, V3 angular, float scale) {
    int32_t* d = &deltas[8 * (size_t)row];
    // i32 wrapping adds, as WGSL atomicAdd on u32 words
    auto add = [](int32_t* word, int32_t v) { atomic_add_u32(reinterpret_cast<uint32_t*>(word), (uint32_t)v); };
    add(d + 0, solver_word(linear.x, scale));
    add(d + 1, solver_word(linear.y, scale));
    add(d + 2, solver_word(linear.z, scale));
    add(d + 3, solver_word(angular.x, scale));
    add(d + 4, solver_word(angular.y, scale));
    add(d + 5, solver_word(angular.z, scale));
}

V3 manifold_arm(const Body& b, const dyn_manifold_point_record& p, bool first) {
    return quat_rotate(b.orientation, first ? rd3(p.local_a) : rd3(p.local_b)) + b.position;
}
float point_momentum_mass(const Body& a, const Body& b, V3 pa, V3 pb, V3 axis) {
    V3 ra = pa - body_com(a);
    V3 rb = pb - body_com(b);
    V3 rax = cross(ra, axis);
    V3 rbx = cross(rb, axis);
    return a.inverse_mass + b.inverse_mass + dot(rax, apply_inverse_inertia(a, rax))
        + dot(rbx, apply_inverse_inertia(b, rbx));
}
void apply_pair_impulse(Body* a, Body* b, V3 pa, V3 pb, V3 impulse) {
    a->velocity = a->velocity - impulse * a->inverse_mass;
    a->angular_velocity = a->angular_velocity - apply_inverse_inertia(*a, cross(pa - body_com(*a), impulse));
    b->velocity = b->velocity + impulse * b->inverse_mass;
    b->angular_velocity = b->angular_velocity + apply_inverse_inertia(*b, cross(pb - body_com(*b), impulse));
}
struct Tangents {
    V3 first, second;
};
Tangents make_tangents(V3 normal) {
    V3 tangent = V3{1.0f, 0.0f, 0.0f};
    if (std::fabs(normal.x) > 0.9f) tangent = V3{0.0f, 1.0f, 0.0f};
    V3 t1 = normalize(cross(normal, tangent));
    V3 t2 = cross(normal, t1);
    return Tangents{t1, t2};
}
// core.wgsl:326-345
float contact_normal_delta(const dyn_contact_record& c, float mass, float truth, float step, float goal, float depth,
                           float speed, float accumulated) {
    if (c.relaxation <= 0.0f) return (goal - speed) / mass;
    float bias = fmaxw(depth / step, goal);
    float drag = 2.0f * c.damping_ratio * c.relaxation / step;
    float softness = c.relaxation * c.relaxation * truth / (step * step);
    float prior = speed - accumulated * truth;
    float wanted = (bias - (1.0f + drag) * prior) / (softness + (1.0f + drag) * truth);
    return truth * (wanted - accumulated) / mass;
}

// solver_contact_block.wgsl:195-233
void warm_contact_block(OracleWorld& w, uint32_t index) {
    const dyn_contact_record& contact = w.contacts[index];
    uint32_t fr = w.blocks[2 * index], sr = w.blocks[2 * index + 1];
    if (!contact_block_resolves(contact)) {
        accumulate(w.velocity_deltas, fr, splat3(0.0f), splat3(0.0f), DYN_SOLVER_VELOCITY_SCALE);
        accumulate(w.velocity_deltas, sr, splat3(0.0f), splat3(0.0f), DYN_SOLVER_VELOCITY_SCALE);
        return;
    }
    Body fl = body_at(w, fr), sl = body_at(w, sr);
    Body first = body_is_inert(fl) ? body_frozen(fl) : fl;
    Body second = body_is_inert(sl) ? body_frozen(sl) : sl;
    V3 normal = rd3(contact.normal);
    Tangents t = make_tangents(normal);
    for (uint32_t pi = 0; pi < contact.point_count; ++pi) {
        const dyn_manifold_point_record& p = contact.points[pi];
        V3 af = manifold_arm(first, p, true);
        V3 as = manifold_arm(second, p, false);
        V3 impulse = normal * p.accumulated_normal + t.first * p.accumulated_tangent_1 + t.second * p.accumulated_tangent_2;
        apply_pair_impulse(&first, &second, af, as, impulse);
    }
    accumulate(w.velocity_deltas, fr, first.velocity - fl.velocity, first.angular_velocity - fl.angular_velocity,
               DYN_SOLVER_VELOCITY_SCALE);
    accumulate(w.velocity_deltas, sr, second.velocity - sl.velocity, second.angular_velocity - sl.angular_velocity,
               DYN_SOLVER_VELOCITY_SCALE);
}

// solver_contact_block.wgsl:6-193 and solver_block_solve.wgsl:39-94
void solve_contact_block(OracleWorld& w, uint32_t index, bool residual) {
    dyn_contact_record& stored = w.contacts[index];
    const dyn_contact_record contact = stored;
    uint32_t fr = w.blocks[2 * index], sr = w.blocks[2 * index + 1];
    auto commit = [&](V3 da, V3 sa, V3 db, V3 sb) {
        accumulate(w.velocity_deltas, fr, da, sa, DYN_SOLVER_VELOCITY_SCALE);
        accumulate(w.velocity_deltas, sr, db, sb, DYN_SOLVER_VELOCITY_SCALE);
        if (!residual) return;
        uint32_t lin = (uint32_t)solver_word(fmaxw(length(da), length(db)), DYN_SOLVER_VELOCITY_SCALE);
        uint32_t ang = (uint32_t)solver_word(fmaxw(length(sa), length(sb)), DYN_SOLVER_VELOCITY_SCALE);
        atomic_max_u32(&w.counters[DYN_COUNTER_SOLVE_LINEAR_RESIDUAL], lin);
        atomic_max_u32(&w.counters[DYN_COUNTER_SOLVE_ANGULAR_RESIDUAL], ang);
    };
    V3 zero = splat3(0.0f);
    if (!contact_block_resolves(contact)) {
        commit(zero, zero, zero, zero);
        return;
    }
    Body pf = body_at(w, fr), ps = body_at(w, sr);
    Body split_f = body_split(pf, (float)std::max(w.block_counts[fr], 1u));
    Body split_s = body_split(ps, (float)std::max(w.block_counts[sr], 1u));
    if (body_is_inert(pf)) {
        pf = body_frozen(pf);
        split_f = body_frozen(split_f);
    }
    if (body_is_inert(ps)) {
        ps = body_frozen(ps);
        split_s = body_frozen(split_s);
    }
    if (body_is_inert(pf) && body_is_inert(ps)) {
        commit(zero, zero, zero, zero);
        return;
    }
    Body first = pf, second = ps;
    V3 normal = rd3(contact.normal);
    Tangents t = make_tangents(normal);
    dyn_contact_record updated = contact;
    V3 reach_f = zero, reach_s = zero;
    for (uint32_t pi = 0; pi < contact.point_count; ++pi) {
        reach_f = reach_f + (manifold_arm(pf, contact.points[pi], true) - body_com(pf));
        reach_s = reach_s + (manifold_arm(ps, contact.points[pi], false) - body_com(ps));
    }
    float point_count = (float)std::max(contact.point_count, 1u);
    float normal_total = 0.0f;
    for (uint32_t pi = 0; pi < contact.point_count; ++pi) {
        normal_total = normal_total + fmaxw(contact.points[pi].accumulated_normal, 0.0f);
    }
    V3 impulses[4] = {zero, zero, zero, zero};
    // manifold_row_mass (solver_contact_block.wgsl:14-29) of every point, then the library's
    // row-mass guard when it is on (DYN_SOLVER_GUARD_ROW_MASS): a block whose points' normalised
    // coupling matrix has an eigenvalue of 1.9 or more (where the reference's Jacobi iteration stops
    // converging at 2) takes count x each point's own coupling instead
    float row_mass[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    V3 arm_fs[4], arm_ss[4];
    for (uint32_t pi = 0; pi < contact.point_count; ++pi) {
        const dyn_manifold_point_record& p = contact.points[pi];
        arm_fs[pi] = cross(manifold_arm(pf, p, true) - body_com(split_f), normal);
        arm_ss[pi] = cross(manifold_arm(ps, p, false) - body_com(split_s), normal);
        row_mass[pi] = point_count * (split_f.inverse_mass + split_s.inverse_mass)
            + dot(apply_inverse_inertia(split_f, cross(reach_f, normal)), arm_fs[pi])
            + dot(apply_inverse_inertia(split_s, cross(reach_s, normal)), arm_ss[pi]);
    }
    if ((w.solver_guard & 1u) && contact.point_count >= 2u) {
        const uint32_t pc = contact.point_count;
        V3 iu[4], iv[4];
        for (uint32_t j = 0; j < pc; ++j) {
            iu[j] = apply_inverse_inertia(split_f, arm_fs[j]);
            iv[j] = apply_inverse_inertia(split_s, arm_ss[j]);
        }
        auto coupling = [&](uint32_t j, uint32_t k) {
            return split_f.inverse_mass + split_s.inverse_mass + dot(arm_fs[j], iu[k]) + dot(arm_ss[j], iv[k]);
        };
        // the row masses stay while every one is positive and 1.9 I - D^-1/2 A D^-1/2 is positive
        // definite (LDL^T pivots, row by row)
        bool converges = true;
        for (uint32_t j = 0; j < pc; ++j) converges = converges && row_mass[j] > 0.0f;
        if (converges) {
            float m[4][4], l[4][4], d[4];
            for (uint32_t j = 0; j < pc; ++j)
                for (uint32_t k = 0; k < pc; ++k)
                    m[j][k] = (j == k ? 1.9f : 0.0f) - coupling(j, k) / std::sqrt(row_mass[j] * row_mass[k]);
            for (uint32_t j = 0; j < pc && converges; ++j) {
                float pivot = m[j][j];
                for (uint32_t k = 0; k < j; ++k) pivot = pivot - l[j][k] * l[j][k] * d[k];
                d[j] = pivot;
                converges = pivot > 0.0f;
                for (uint32_t i = j + 1; i < pc && converges; ++i) {
                    float x = m[i][j];
                    for (uint32_t k = 0; k < j; ++k) x = x - l[i][k] * l[j][k] * d[k];
                    l[i][j] = x / pivot;
                }
            }
        }
        if (!converges)
            for (uint32_t j = 0; j < pc; ++j) row_mass[j] = point_count * coupling(j, j);
    }
    for (uint32_t pi = 0; pi < contact.point_count; ++pi) {
        const dyn_manifold_point_record& p = contact.points[pi];
        V3 af = manifold_arm(pf, p, true);
        V3 as = manifold_arm(ps, p, false);
        float acc_n = p.accumulated_normal;
        float acc_t1 = p.accumulated_tangent_1;
        float acc_t2 = p.accumulated_tangent_2;
        float normal_speed = dot(relative_velocity(pf, ps, af, as), normal);
        float normal_mass = row_mass[pi];
        float normal_truth = point_momentum_mass(pf, ps, af, as, normal);
        float delta = contact_normal_delta(contact, normal_mass, normal_truth, w.params.dt,
                                           w.target_speeds[4 * (size_t)index + pi], p.depth, normal_speed, acc_n);
        float next_normal = fmaxw(0.0f, acc_n + delta);
        uint8_t flags = acc_n + delta > 0.0f ? 1u : 0u;
        impulses[pi] = impulses[pi] + normal * (next_normal - acc_n);
        acc_n = next_normal;
        float friction_limit = contact.friction * acc_n;
        float t1_mass = point_momentum_mass(split_f, split_s, af, as, t.first) * (float)std::max(contact.point_count, 1u);
        float t1_speed = dot(relative_velocity(pf, ps, af, as), t.first);
        const float want_t1 = acc_t1 - t1_speed / t1_mass;
        float next_t1 = clampw(want_t1, -friction_limit, friction_limit);
        flags |= want_t1 > friction_limit ? 2u : (want_t1 < -friction_limit ? 4u : 0u);
        impulses[pi] = impulses[pi] + t.first * (next_t1 - acc_t1);
        acc_t1 = next_t1;
        float t2_mass = point_momentum_mass(split_f, split_s, af, as, t.second) * (float)std::max(contact.point_count, 1u);
        float t2_speed = dot(relative_velocity(pf, ps, af, as), t.second);
        const float remaining_sq = friction_limit * friction_limit - acc_t1 * acc_t1;
        float remaining = std::sqrt(fmaxw(remaining_sq, 0.0f));
        const float want_t2 = acc_t2 - t2_speed / t2_mass;
        float next_t2 = clampw(want_t2, -remaining, remaining);
        // the device adjoint's rule: below 5 % of the friction limit the tangent-2 limit is locally constant
        flags |= (remaining_sq > 0.0f && remaining > 0.05f * friction_limit) ? 8u : 0u;
        flags |= want_t2 > remaining ? 16u : (want_t2 < -remaining ? 32u : 0u);
        {
            const dyn_step_params& sp = w.params;
            const size_t c = w.contacts.size();
            w.solve_flags[(((size_t)w.flag_substep * sp.solve_iterations + w.flag_iteration) * c + index) * 4 + pi] = flags;
        }
        impulses[pi] = impulses[pi] + t.second * (next_t2 - acc_t2);
        acc_t2 = next_t2;
        updated.points[pi].accumulated_normal = acc_n;
        updated.points[pi].accumulated_tangent_1 = acc_t1;
        updated.points[pi].accumulated_tangent_2 = acc_t2;
    }
    for (uint32_t pi = 0; pi < contact.point_count; ++pi) {
        V3 af = manifold_arm(pf, contact.points[pi], true);
        V3 as = manifold_arm(ps, contact.points[pi], false);
        apply_pair_impulse(&first, &second, af, as, impulses[pi]);
    }
    V3 rel_spin = second.angular_velocity - first.angular_velocity;
    V3 planar_spin = rel_spin - normal * dot(rel_spin, normal);
    float planar_len = length(planar_spin);
    if (planar_len > 1e-6f) {
        V3 axis = planar_spin / planar_len;
        float mass = dot(axis, apply_inverse_inertia(split_f, axis)) + dot(axis, apply_inverse_inertia(split_s, axis));
        if (mass > 0.0f) {
            float limit = contact.rolling_friction * normal_total;
            float applied = clampw(-planar_len / mass, -limit, limit);
            first.angular_velocity = first.angular_velocity - apply_inverse_inertia(first, axis * applied);
            second.angular_velocity = second.angular_velocity + apply_inverse_inertia(second, axis * applied);
        }
    }
    float twist = dot(rel_spin, normal);
    if (std::fabs(twist) > 1e-6f) {
        float mass = dot(normal, apply_inverse_inertia(split_f, normal)) + dot(normal, apply_inverse_inertia(split_s, normal));
        if (mass > 0.0f) {
            float limit = contact.spin_friction * normal_total;
            float applied = clampw(-twist / mass, -limit, limit);
            first.angular_velocity = first.angular_velocity - apply_inverse_inertia(first, normal * applied);
            second.angular_velocity = second.angular_velocity + apply_inverse_inertia(second, normal * applied);
        }
    }
    stored = updated;
    commit(first.velocity - pf.velocity, first.angular_velocity - pf.angular_velocity, second.velocity - ps.velocity,
           second.angular_velocity - ps.angular_velocity);
}

// solver_block_apply.wgsl:7-29
void block_apply(OracleWorld& w) {
    if (!w.solver_rows.empty()) w.solver_rounds += 1;
    const size_t rows = w.solver_rows.size();
#pragma omp parallel for schedule(static)
    for (size_t r = 0; r < rows; ++r) {
        const uint32_t row = w.solver_rows[r];
        int32_t* d = &w.velocity_deltas[8 * (size_t)row];
        V3 linear = V3{solver_value(d[0], DYN_SOLVER_VELOCITY_SCALE), solver_value(d[1], DYN_SOLVER_VELOCITY_SCALE),
                       solver_value(d[2], DYN_SOLVER_VELOCITY_SCALE)};
        V3 angular = V3{solver_value(d[3], DYN_SOLVER_VELOCITY_SCALE), solver_value(d[4], DYN_SOLVER_VELOCITY_SCALE),
                        solver_value(d[5], DYN_SOLVER_VELOCITY_SCALE)};
        for (int k = 0; k < 6; ++k) d[k] = 0;
        if (veq(linear, splat3(0.0f)) && veq(angular, splat3(0.0f))) continue;
        dyn_body_state_record& s = w.states[row];
        // (rows are distinct: each solver row is claimed once)
        wr3(s.velocity, rd3(s.velocity) + linear);
        wr3(s.angular_velocity, rd3(s.angular_velocity) + angular);
    }
}

// substep_integrate.wgsl:15-76 (no force fields)
void substep_integrate(OracleWorld& w) {
    w.solver_rounds = 0;
    const dyn_step_params& p = w.params;
    float h = p.substep_dt;
    const size_t live = w.live.size();
#pragma omp parallel for schedule(static)
    for (size_t r = 0; r < live; ++r) {
        const uint32_t row = w.live[r];
        const dyn_body_descriptor_record& d = w.descs[row];
        if (!body_simulates_d(d.inverse_mass, d.flags)) continue;
        dyn_body_state_record& s = w.states[row];
        V4 q = rd4(s.orientation);
        V3 acceleration = V3{p.gravity[0], p.gravity[1], p.gravity[2]} * d.gravity_scale + rd3(s.force) * d.inverse_mass;
        V3 spin = rd3(s.angular_velocity);
        V3 velocity = rd3(s.velocity) + acceleration * h;
        // gyroscopic_spin
        V3 gyro = spin;
        const float* I = d.inertia;
        bool isotropic = I[1] == 0.0f && I[2] == 0.0f && I[4] == 0.0f && I[0] == I[3] && I[3] == I[5];
        if (!isotropic) {
            V3 body_spin = quat_rotate(quat_conjugate(q), spin);
            V3 momentum = symmetric_apply(I, body_spin);
            if (!veq(cross(body_spin, momentum), splat3(0.0f))) {
                V3 solved = momentum;
                for (int it = 0; it < 4; ++it) {
                    V3 midpoint = 0.5f * (momentum + solved);
                    solved = rotate_about(-symmetric_apply(d.inverse_inertia, midpoint) * h, momentum);
                }
                gyro = quat_rotate(q, symmetric_apply(d.inverse_inertia, solved));
            }
        }
        V3 angular = gyro + apply_inverse_inertia_of(d.inverse_inertia, q, rd3(s.torque) * h);
        float speed = length(velocity);
        if (speed > p.max_velocity) velocity = velocity * (p.max_velocity / speed);
        float spin_speed = length(angular);
        if (spin_speed > p.max_angular_velocity) angular = angular * (p.max_angular_velocity / spin_speed);
        if (!w.integrate_flags.empty()) {
            w.integrate_flags[(size_t)w.flag_substep * w.states.size() + row] =
                (uint8_t)((speed > p.max_velocity ? 1u : 0u) | (spin_speed > p.max_angular_velocity ? 2u : 0u));
        }
        velocity = velocity / (1.0f + d.linear_damping * h);
        angular = angular / (1.0f + d.angular_damping * h);
        wr3(s.velocity, velocity);
        wr3(s.angular_velocity, angular);
    }
}

// substep_advance.wgsl:6-13
void substep_advance(OracleWorld& w) {
    float h = w.params.substep_dt;
    const size_t live = w.live.size();
#pragma omp parallel for schedule(static)
    for (size_t r = 0; r < live; ++r) {
        dyn_body_state_record& s = w.states[w.live[r]];
        wr3(s.position, rd3(s.position) + rd3(s.velocity) * h);
        V3 av = rd3(s.angular_velocity);
        V4 spin = V4{av.x, av.y, av.z, 0.0f};
        V4 q = rd4(s.orientation);
        wr4(s.orientation, normalize(q + 0.5f * h * quat_mul(spin, q)));
    }
}

// position_correction.wgsl:5-46 + position_block.wgsl:11-33
void position_block(OracleWorld& w) {
    uint32_t c = (uint32_t)w.contacts.size();
#pragma omp parallel for schedule(dynamic, 256)
    for (uint32_t index = 0; index < c; ++index) {
        const dyn_contact_record& contact = w.contacts[index];
        if (!contact_block_resolves(contact) || contact.relaxation > 0.0f) continue;
        uint32_t fr = w.blocks[2 * index], sr = w.blocks[2 * index + 1];
        Body fl = body_at(w, fr), sl = body_at(w, sr);
        Body first = body_is_inert(fl) ? body_frozen(fl) : fl;
        Body second = body_is_inert(sl) ? body_frozen(sl) : sl;
        V3 normal = rd3(contact.normal);
        float resolved = dot(normal, w.resolution[sr] - w.resolution[fr]);
        V3 total = splat3(0.0f);
        uint32_t contributing = 0;
        uint8_t corrects[4] = {0u, 0u, 0u, 0u};
        for (uint32_t pi = 0; pi < contact.point_count; ++pi) {
            float error = fmaxw(contact.points[pi].depth - w.params.slop - resolved, 0.0f);
            if (error <= 0.0f) continue;
            float k = first.inverse_mass + second.inverse_mass;
            if (k == 0.0f) continue;
            total = total + normal * (w.params.relaxation * error / k);
            contributing += 1;
            corrects[pi] = 1u;
        }
        if (contributing == 0u) continue;
        V3 correction = total / (float)contributing;
        V3 lin_f = -correction * first.inverse_mass;
        V3 lin_s = correction * second.inverse_mass;
        // correction.wgsl:18-31 pair_holds
        bool holds = dot(lin_f, lin_f) > 0.0f || dot(lin_s, lin_s) > 0.0f;
        if (!holds) continue;
        for (uint32_t pi = 0; pi < 4; ++pi) {
            w.position_flags[(((size_t)w.flag_substep * w.params.position_iterations + w.flag_iteration) * c + index) * 4 + pi] =
                corrects[pi];
        }
        atomic_add_u32(&w.contributions[fr], 1u);
        atomic_add_u32(&w.contributions[sr], 1u);
        accumulate(w.position_deltas, fr, lin_f, splat3(0.0f), DYN_SOLVER_POSITION_SCALE);
        accumulate(w.position_deltas, sr, lin_s, splat3(0.0f), DYN_SOLVER_POSITION_SCALE);
    }
}

// position_apply.wgsl:12-27
void position_apply(OracleWorld& w) {
    const size_t rows = w.solver_rows.size();
#pragma omp parallel for schedule(static)
    for (size_t r = 0; r < rows; ++r) {
        const uint32_t row = w.solver_rows[r];
        uint32_t contributing = w.contributions[row];
        w.contributions[row] = 0;
        int32_t* d = &w.position_deltas[8 * (size_t)row];
        V3 linear = V3{solver_value(d[0], DYN_SOLVER_POSITION_SCALE), solver_value(d[1], DYN_SOLVER_POSITION_SCALE),
                       solver_value(d[2], DYN_SOLVER_POSITION_SCALE)};
        V3 angular = V3{solver_value(d[3], DYN_SOLVER_POSITION_SCALE), solver_value(d[4], DYN_SOLVER_POSITION_SCALE),
                        solver_value(d[5], DYN_SOLVER_POSITION_SCALE)};
        for (int k = 0; k < 6; ++k) d[k] = 0;
        if (contributing == 0u) continue;
        V3 applied_linear = linear / (float)contributing;
        V3 applied_angular = angular / (float)contributing;
        dyn_body_state_record& s = w.states[row];
        wr3(s.position, rd3(s.position) + applied_linear);
        V3 ha = applied_angular * 0.5f;
        wr4(s.orientation, normalize(quat_mul(V4{ha.x, ha.y, ha.z, 1.0f}, rd4(s.orientation))));
        w.resolution[row] = w.resolution[row] + applied_linear;
    }
}


// ---- ball joints (joint_velocity.wgsl, joint_solve.wgsl, joint_position.wgsl, joint_correction.wgsl) ----

// schedule.rs:105-296 solve_order: components, layers, and the component order of the plan.
uint32_t plan_root(std::vector<uint32_t>& roots, uint32_t row) {
    while (roots[row] != row) {
        roots[row] = roots[roots[row]];
        row = roots[row];
    }
    return row;
}
void plan_joint_order(OracleWorld& w) {
    const uint32_t none = 0xFFFFFFFFu;
    const uint32_t joints = (uint32_t)w.joint_descs.size();
    const uint32_t rows_n = (uint32_t)w.states.size();
    w.plan_rows.clear();
    w.plan_layers.clear();
    w.plan_components.clear();
    if (joints == 0) return;
    std::vector<uint32_t> a(joints), b(joints);
    for (uint32_t j = 0; j < joints; ++j) {
        a[j] = w.joint_rows[j].first_row;
        b[j] = w.joint_rows[j].second_row;
    }
    std::vector<bool> anchor(rows_n, false);
    std::vector<uint32_t> roots(rows_n);
    for (uint32_t i = 0; i < rows_n; ++i) roots[i] = i;
    for (uint32_t j = 0; j < joints; ++j) {
        if (!body_simulates_d(w.descs[a[j]].inverse_mass, w.descs[a[j]].flags)) anchor[a[j]] = true;
        if (!body_simulates_d(w.descs[b[j]].inverse_mass, w.descs[b[j]].flags)) anchor[b[j]] = true;
        uint32_t fr = plan_root(roots, a[j]), sr = plan_root(roots, b[j]);
        uint32_t root = std::min(fr, sr);
        roots[fr] = root;
        roots[sr] = root;
    }
    std::vector<uint32_t> roots_of(joints);
    for (uint32_t j = 0; j < joints; ++j) roots_of[j] = plan_root(roots, a[j]);
    std::vector<bool> anchored(rows_n, false);
    std::vector<uint32_t> head_of(rows_n, none);
    for (uint32_t j = 0; j < joints; ++j) {
        uint32_t root = roots_of[j];
        if (anchor[a[j]] || anchor[b[j]]) anchored[root] = true;
        head_of[root] = std::min(head_of[root], std::min(a[j], b[j]));
    }
    std::vector<std::vector<uint32_t>> adjacency(rows_n);
    for (uint32_t j = 0; j < joints; ++j) {
        adjacency[a[j]].push_back(b[j]);
        adjacency[b[j]].push_back(a[j]);
    }
    std::vector<uint32_t> depth(rows_n, none), frontier;
    for (uint32_t body = 0; body < rows_n; ++body) {
        if (anchor[body]) {
            depth[body] = 0;
            frontier.push_back(body);
        }
    }
    for (uint32_t root = 0; root < rows_n; ++root) {
        if (head_of[root] != none && !anchored[root]) {
            depth[head_of[root]] = 0;
            frontier.push_back(head_of[root]);
        }
    }
    for (size_t cursor = 0; cursor < frontier.size(); ++cursor) {
        uint32_t body = frontier[cursor];
        for (uint32_t neighbor : adjacency[body]) {
            if (depth[neighbor] == none) {
                depth[neighbor] = depth[body] + 1;
                frontier.push_back(neighbor);
            }
        }
    }
    struct Key {
        uint32_t depth, root, row;
    };
    std::vector<Key> settled(joints);
    for (uint32_t j = 0; j < joints; ++j) settled[j] = Key{std::max(depth[a[j]], depth[b[j]]), roots_of[j], j};
    std::sort(settled.begin(), settled.end(), [](const Key& x, const Key& y) {
        return x.depth != y.depth ? x.depth < y.depth : (x.root != y.root ? x.root < y.root : x.row < y.row);
    });
    std::vector<uint32_t> held_layer(rows_n, 0);
    std::vector<std::array<uint32_t, 3>> held;  // (root, layer, row)
    for (const Key& k : settled) {
        uint32_t layer = std::max(held_layer[a[k.row]], held_layer[b[k.row]]) + 1;
        held_layer[a[k.row]] = layer;
        held_layer[b[k.row]] = layer;
        held.push_back({roots_of[k.row], layer, k.row});
    }
    std::sort(held.begin(), held.end());
    struct Component {
        uint32_t first_layer, layers, first_row, head, lanes;
    };
    std::vector<uint32_t> rows, layers;
    std::vector<Component> components;
    size_t index = 0;
    while (index < held.size()) {
        uint32_t root = held[index][0];
        Component c{(uint32_t)(layers.size() / 2), 0, (uint32_t)rows.size(), none, 0};
        uint32_t lanes = 0;
        while (index < held.size() && held[index][0] == root) {
            uint32_t layer = held[index][1];
            size_t first = rows.size();
            while (index < held.size() && held[index][0] == root && held[index][1] == layer) {
                uint32_t row = held[index][2];
                c.head = std::min(c.head, std::min(a[row], b[row]));
                rows.push_back(row);
                ++index;
            }
            uint32_t count = (uint32_t)(rows.size() - first);
            lanes = std::max(lanes, count);
            layers.push_back((uint32_t)first);
            layers.push_back(count);
            c.layers += 1;
        }
        uint32_t p2 = 1;
        while (p2 < lanes) p2 <<= 1;
        c.lanes = std::min(std::max(p2, 1u), 64u);
        components.push_back(c);
    }
    std::stable_sort(components.begin(), components.end(), [](const Component& x, const Component& y) {
        if (x.lanes != y.lanes) return x.lanes > y.lanes;
        if (x.layers != y.layers) return x.layers > y.layers;
        return x.head < y.head;
    });
    for (const Component& c : components) {
        w.plan_components.push_back((uint32_t)(w.plan_layers.size() / 2));
        w.plan_components.push_back(c.layers);
        uint32_t cursor = c.first_row;
        for (uint32_t layer = c.first_layer; layer < c.first_layer + c.layers; ++layer) {
            uint32_t count = layers[2 * layer + 1];
            w.plan_layers.push_back((uint32_t)w.plan_rows.size());
            w.plan_layers.push_back(count);
            for (uint32_t i = 0; i < count; ++i) w.plan_rows.push_back(rows[cursor + i]);
            cursor += count;
        }
    }
}

V3 world_axis(uint32_t i) { return V3{i == 0 ? 1.0f : 0.0f, i == 1 ? 1.0f : 0.0f, i == 2 ? 1.0f : 0.0f}; }
V3 constraint_anchor(const Body& b, V3 local) { return b.position + quat_rotate(b.orientation, local); }
void store_velocity(OracleWorld& w, uint32_t row, const Body& b) {
    wr3(w.states[row].velocity, b.velocity);
    wr3(w.states[row].angular_velocity, b.angular_velocity);
}

// joint_solve.wgsl:803-832 warm_joint (ball rows of warm_constraint_rows :754-766)
void joint_warm(OracleWorld& w, uint32_t j) {
    const dyn_constraint_runtime_record& rt = w.joint_runtime[j];
    if (rt.broken != 0u) return;
    const dyn_constraint_descriptor_record& c = w.joint_descs[j];
    const dyn_constraint_rows_record& r = w.joint_rows[j];
    Body first_loaded = body_at(w, r.first_row), second_loaded = body_at(w, r.second_row);
    Body first = body_is_inert(first_loaded) ? body_frozen(first_loaded) : first_loaded;
    Body second = body_is_inert(second_loaded) ? body_frozen(second_loaded) : second_loaded;
    if (c.flags & DYN_CONSTRAINT_WARM_START) {
        V3 anchor_a = constraint_anchor(first, rd3(c.anchor_a));
        V3 anchor_b = constraint_anchor(second, rd3(c.anchor_b));
        for (uint32_t i = 0; i < 3; ++i) apply_pair_impulse(&first, &second, anchor_a, anchor_b, world_axis(i) * rt.accumulated[i]);
    }
    store_velocity(w, r.first_row, first);
    store_velocity(w, r.second_row, second);
}

// joint_solve.wgsl:236-267, 419-430 solve_joint for a ball joint; solve_point_row :96-128
void joint_solve(OracleWorld& w, uint32_t j, bool residual) {
    dyn_constraint_runtime_record& rt = w.joint_runtime[j];
    const dyn_constraint_descriptor_record& c = w.joint_descs[j];
    const dyn_constraint_rows_record& r = w.joint_rows[j];
    float accumulated[DYN_CONSTRAINT_ACCUMULATOR_SLOTS];
    for (uint32_t i = 0; i < DYN_CONSTRAINT_ACCUMULATOR_SLOTS; ++i)
        accumulated[i] = (c.flags & DYN_CONSTRAINT_WARM_START) ? rt.accumulated[i] : 0.0f;
    if (rt.broken != 0u) return;
    Body first_loaded = body_at(w, r.first_row), second_loaded = body_at(w, r.second_row);
    if (body_is_inert(first_loaded) && body_is_inert(second_loaded)) return;
    Body first = body_is_inert(first_loaded) ? body_frozen(first_loaded) : first_loaded;
    Body second = body_is_inert(second_loaded) ? body_frozen(second_loaded) : second_loaded;
    const Body mass_first = first, mass_second = second;
    V3 anchor_a = constraint_anchor(first, rd3(c.anchor_a));
    V3 anchor_b = constraint_anchor(second, rd3(c.anchor_b));
    V3 linear_first{0, 0, 0}, angular_first{0, 0, 0}, linear_second{0, 0, 0}, angular_second{0, 0, 0};
    for (uint32_t i = 0; i < 3; ++i) {
        V3 axis = world_axis(i);
        float k = point_momentum_mass(mass_first, mass_second, anchor_a, anchor_b, axis);
        if (k > 0.0f) {
            Body row_first = first, row_second = second;
            V3 velocity = relative_velocity(first, second, anchor_a, anchor_b);
            float jacobian_speed = dot(velocity, axis);
            float next = accumulated[i] - jacobian_speed / k;
            float applied = next - accumulated[i];
            apply_pair_impulse(&first, &second, anchor_a, anchor_b, axis * applied);
            accumulated[i] = next;
            V3 impulse = axis * accumulated[i];
            linear_first = linear_first + (-impulse);
            linear_second = linear_second + impulse;
            angular_first = angular_first + cross(anchor_a - body_com(row_first), -impulse);
            angular_second = angular_second + cross(anchor_b - body_com(row_second), impulse);
        }
    }
    if (c.flags & DYN_CONSTRAINT_HAS_BREAK) {
        float force = length(linear_second) / w.params.dt;
        float torque = length(angular_second) / w.params.dt;
        if ((c.break_force > 0.0f && force > c.break_force) || (c.break_torque > 0.0f && torque > c.break_torque)) rt.broken = 1u;
    }
    for (uint32_t i = 0; i < DYN_CONSTRAINT_ACCUMULATOR_SLOTS; ++i) rt.accumulated[i] = accumulated[i];
    std::memset(&rt.reaction, 0, sizeof(rt.reaction));
    wr3(rt.reaction.linear_first, linear_first);
    wr3(rt.reaction.angular_first, angular_first);
    wr3(rt.reaction.linear_second, linear_second);
    wr3(rt.reaction.angular_second, angular_second);
    store_velocity(w, r.first_row, first);
    store_velocity(w, r.second_row, second);
    if (!residual) return;
    uint32_t lin = (uint32_t)solver_word(fmaxw(length(first.velocity - first_loaded.velocity),
                                               length(second.velocity - second_loaded.velocity)),
                                         DYN_SOLVER_VELOCITY_SCALE);
    uint32_t ang = (uint32_t)solver_word(fmaxw(length(first.angular_velocity - first_loaded.angular_velocity),
                                               length(second.angular_velocity - second_loaded.angular_velocity)),
                                         DYN_SOLVER_VELOCITY_SCALE);
    w.counters[DYN_COUNTER_SOLVE_LINEAR_RESIDUAL] = std::max(w.counters[DYN_COUNTER_SOLVE_LINEAR_RESIDUAL], lin);
    w.counters[DYN_COUNTER_SOLVE_ANGULAR_RESIDUAL] = std::max(w.counters[DYN_COUNTER_SOLVE_ANGULAR_RESIDUAL], ang);
}

// joint_position.wgsl:18-36 project over joint_correction.wgsl:5-27, 85-90 (ball: three point rows)
void apply_correction(Body* b, V3 linear, V3 angular) {
    b->position = b->position + linear;
    V3 half = angular * 0.5f;
    b->orientation = normalize(quat_mul(V4{half.x, half.y, half.z, 1.0f}, b->orientation));
}
void joint_project(OracleWorld& w, uint32_t j) {
    const dyn_constraint_descriptor_record& c = w.joint_descs[j];
    const dyn_constraint_rows_record& r = w.joint_rows[j];
    if (w.joint_runtime[j].broken != 0u) return;
    Body first_loaded = body_at(w, r.first_row), second_loaded = body_at(w, r.second_row);
    Body first = body_is_inert(first_loaded) ? body_frozen(first_loaded) : first_loaded;
    Body second = body_is_inert(second_loaded) ? body_frozen(second_loaded) : second_loaded;
    const float scale = w.params.relaxation;
    V3 zero{0.0f, 0.0f, 0.0f};
    V3 total_first = zero, total_first_angular = zero, total_second = zero, total_second_angular = zero;
    for (uint32_t i = 0; i < 3; ++i) {
        V3 axis = world_axis(i);
        V3 point_a = constraint_anchor(first, rd3(c.anchor_a));
        V3 point_b = constraint_anchor(second, rd3(c.anchor_b));
        V3 linear_first = zero, linear_second = zero;
        float k = first.inverse_mass + second.inverse_mass;  // linear_momentum_mass
        if (k > 0.0f) {
            float magnitude = scale * (dot(point_b - point_a, axis) - 0.0f) / k;
            linear_first = axis * (magnitude * first.inverse_mass);
            linear_second = axis * (-magnitude * second.inverse_mass);
        }
        apply_correction(&first, linear_first, zero);
        apply_correction(&second, linear_second, zero);
        total_first = total_first + linear_first;
        total_first_angular = total_first_angular + zero;
        total_second = total_second + linear_second;
        total_second_angular = total_second_angular + zero;
    }
    bool holds = dot(total_first, total_first) > 0.0f || dot(total_first_angular, total_first_angular) > 0.0f ||
                 dot(total_second, total_second) > 0.0f || dot(total_second_angular, total_second_angular) > 0.0f;
    if (!holds) return;
    dyn_body_state_record& sa = w.states[r.first_row];
    dyn_body_state_record& sb = w.states[r.second_row];
    Body fa = load_body(sa, w.descs[r.first_row]), fb = load_body(sb, w.descs[r.second_row]);
    apply_correction(&fa, total_first, total_first_angular);
    apply_correction(&fb, total_second, total_second_angular);
    wr3(sa.position, fa.position);
    wr4(sa.orientation, fa.orientation);
    wr3(sb.position, fb.position);
    wr4(sb.orientation, fb.orientation);
    w.resolution[r.first_row] = w.resolution[r.first_row] + total_first;
    w.resolution[r.second_row] = w.resolution[r.second_row] + total_second;
}

// joint_velocity.wgsl:24-54 / joint_position.wgsl:30-61: every component, a forward and a backward
// sweep over its layers. Components and the joints of a layer touch disjoint bodies, so visiting
// them in sequence gives what the parallel lanes give.
enum class JointWalk { Warm, Solve, Project };
void walk_joints(OracleWorld& w, JointWalk mode, bool residual) {
    for (size_t c = 0; c + 1 < w.plan_components.size(); c += 2) {
        uint32_t offset = w.plan_components[c], count = w.plan_components[c + 1];
        for (uint32_t sweep = 0; sweep < 2; ++sweep) {
            for (uint32_t step = 0; step < count; ++step) {
                uint32_t layer = sweep == 0 ? offset + step : offset + count - 1 - step;
                uint32_t first = w.plan_layers[2 * layer], n = w.plan_layers[2 * layer + 1];
                for (uint32_t i = 0; i < n; ++i) {
                    uint32_t j = w.plan_rows[first + i];
                    if (mode == JointWalk::Warm) joint_warm(w, j);
                    else if (mode == JointWalk::Solve) joint_solve(w, j, residual);
                    else joint_project(w, j);
                }
            }
        }
    }
}

// solver.rs:304-333 SolveSubsteps.record
void solve_substeps(OracleWorld& w) {
    uint32_t c = (uint32_t)w.contacts.size();
    const size_t n = w.states.size();
    const dyn_step_params& sp = w.params;
    if (w.keep_snapshots) {
        w.snap_pose.assign((size_t)sp.substeps * n * 13, 0.0f);
        w.snap_vel.assign((size_t)sp.substeps * sp.solve_iterations * n * 6, 0.0f);
        w.snap_acc.assign((size_t)sp.substeps * sp.solve_iterations * c * 12, 0.0f);
        w.snap_res.assign((size_t)sp.substeps * sp.position_iterations * n * 3, 0.0f);
    }
    for (uint32_t substep = 0; substep < w.params.substeps; ++substep) {
        w.flag_substep = substep;
        if (w.keep_snapshots) {
            for (size_t r = 0; r < n; ++r) {
                float* o = &w.snap_pose[((size_t)substep * n + r) * 13];
                for (int k = 0; k < 3; ++k) o[k] = w.states[r].position[k];
                for (int k = 0; k < 4; ++k) o[3 + k] = w.states[r].orientation[k];
                for (int k = 0; k < 3; ++k) o[7 + k] = w.states[r].velocity[k];
                for (int k = 0; k < 3; ++k) o[10 + k] = w.states[r].angular_velocity[k];
            }
        }
        substep_integrate(w);
        if (substep == 0) {
            walk_joints(w, JointWalk::Warm, false);
#pragma omp parallel for schedule(dynamic, 256)
            for (uint32_t i = 0; i < c; ++i) warm_contact_block(w, i);
            block_apply(w);
        }
        for (uint32_t it = 0; it < w.params.solve_iterations; ++it) {
            w.flag_iteration = it;
            if (w.keep_snapshots) {
                for (size_t r = 0; r < n; ++r) {
                    float* o = &w.snap_vel[(((size_t)substep * sp.solve_iterations + it) * n + r) * 6];
                    for (int k = 0; k < 3; ++k) o[k] = w.states[r].velocity[k];
                    for (int k = 0; k < 3; ++k) o[3 + k] = w.states[r].angular_velocity[k];
                }
                for (size_t i = 0; i < c; ++i) {
                    for (uint32_t pi = 0; pi < 4; ++pi) {
                        float* o = &w.snap_acc[((((size_t)substep * sp.solve_iterations + it) * c + i) * 4 + pi) * 3];
                        o[0] = w.contacts[i].points[pi].accumulated_normal;
                        o[1] = w.contacts[i].points[pi].accumulated_tangent_1;
                        o[2] = w.contacts[i].points[pi].accumulated_tangent_2;
                    }
                }
            }
            bool residual = w.solver_rounds == w.params.solve_iterations;
            walk_joints(w, JointWalk::Solve, residual);
#pragma omp parallel for schedule(dynamic, 256)
            for (uint32_t i = 0; i < c; ++i) solve_contact_block(w, i, residual);
            block_apply(w);
        }
        substep_advance(w);
        for (uint32_t it = 0; it < w.params.position_iterations; ++it) {
            w.flag_iteration = it;
            if (w.keep_snapshots) {
                for (size_t r = 0; r < n; ++r) {
                    float* o = &w.snap_res[(((size_t)substep * sp.position_iterations + it) * n + r) * 3];
                    o[0] = w.resolution[r].x;
                    o[1] = w.resolution[r].y;
                    o[2] = w.resolution[r].z;
                }
            }
            walk_joints(w, JointWalk::Project, false);
            position_block(w);
            position_apply(w);
        }
    }
}

// island_sleep.wgsl:10-29 (core.wgsl:218-227 freeze_body)
// ---- continuous collision: crates/dynamis-rigid/shaders/ccd_sweep.wgsl, ccd_apply.wgsl ----

// core.wgsl:149-163
V4 quat_slerp(V4 a, V4 b, float t) {
    float cosine = dot(a, b);
    if (cosine < 0.0f) {
        b = -b;
        cosine = -cosine;
    }
    if (cosine > 0.9995f) return normalize(a + (b - a) * t);
    float angle = oacos(clampw(cosine, -1.0f, 1.0f));
    float sine = osin(angle);
    return (a * (osin((1.0f - t) * angle) / sine)) + (b * (osin(t * angle) / sine));
}
// core.wgsl:165-168
float quat_angle(V4 a, V4 b) { return 2.0f * oacos(std::fabs(clampw(dot(a, b), -1.0f, 1.0f))); }

struct SweepPose {
    Body body;
    V3 prev_position;
    V4 prev_orientation;
};
SweepPose sweep_body(const OracleWorld& w, uint32_t row) {
    const dyn_body_state_record& s = w.states[row];
    return SweepPose{body_at(w, row), rd3(s.prev_position), rd4(s.prev_orientation)};
}
// ccd_sweep.wgsl:40-45
WorldShape sweep_collider(const SweepPose& s, const dyn_collider_record& c, float t) {
    V3 position = s.prev_position + (s.body.position - s.prev_position) * t;
    return world_collider(position, quat_slerp(s.prev_orientation, s.body.orientation, t), c);
}
// ccd_sweep.wgsl:47-54
float sweep_radius(const OracleWorld& w, const Body& b, const dyn_collider_record& c) {
    if (c.kind == DYN_SHAPE_PLANE) return 0.0f;
    Aabb bounds = world_aabb_of(w.shapes, world_collider(b.position, b.orientation, c));
    V3 center = b.position + quat_rotate(b.orientation, rd3(c.local_offset));
    return length((bounds.max - bounds.min) * 0.5f) + length(center - body_com(b));
}
// ccd_sweep.wgsl:56-61: (travel, spin)
void sweep_reach(const OracleWorld& w, const SweepPose& s, const dyn_collider_record& c, float* travel, float* spin) {
    *travel = length(s.body.position - s.prev_position);
    *spin = quat_angle(s.prev_orientation, s.body.orientation) * sweep_radius(w, s.body, c);
}
// ccd_sweep.wgsl:63-69
ShapeHit plane_convex_gap(const OracleWorld& w, const WorldShape& plane, const WorldShape& convex) {
    V3 normal = quat_rotate(plane.rotation, V3{0.0f, 1.0f, 0.0f});
    float side = dot(convex.center - plane.center, normal);
    V3 facing = side < 0.0f ? -normal : normal;
    float extent = dot(support(w.shapes, convex, facing) - convex.center, facing);
    return ShapeHit{std::fabs(side) - extent, convex.center + facing * extent, facing, DYN_NO_TRIANGLE};
}
// ccd_sweep.wgsl:71-98 (triangle scenes are refused at scene set-up: no hit)
ShapeHit pair_gap(const OracleWorld& w, const WorldShape& first, const WorldShape& second) {
    if (first.kind == DYN_SHAPE_PLANE) {
        ShapeHit swapped = plane_convex_gap(w, first, second);
        return ShapeHit{swapped.distance, swapped.point, -swapped.normal, DYN_NO_TRIANGLE};
    }
    if (second.kind == DYN_SHAPE_PLANE) return plane_convex_gap(w, second, first);
    if (shape_world_geometry(first.kind) || shape_world_geometry(second.kind))
        return ShapeHit{kNoHit, splat3(0.0f), splat3(0.0f), DYN_NO_TRIANGLE};
    return convex_hit(w.shapes, first, second);
}

struct SweepHit {
    float time;
    V3 normal, point;
};
// ccd_sweep.wgsl:100-147
SweepHit rigid_sweep(const OracleWorld& w, const SweepPose& moving, const dyn_collider_record& mc, const SweepPose& other,
                     const dyn_collider_record& oc) {
    const SweepHit none{1.0f, V3{0.0f, 1.0f, 0.0f}, splat3(0.0f)};
    if (!body_has_ccd(moving.body)) return none;
    float free_travel_len = 0.0f, free_spin = 0.0f, other_travel_len = 0.0f, other_spin = 0.0f;
    sweep_reach(w, moving, mc, &free_travel_len, &free_spin);
    bool other_movable = body_moves(other.body);
    if (other_movable) sweep_reach(w, other, oc, &other_travel_len, &other_spin);
    float closing_floor = free_spin + other_spin;
    if (free_travel_len + closing_floor + other_travel_len <= 0.0f) return none;
    V3 free_travel = moving.body.position - moving.prev_position;
    V3 other_travel = other_movable ? other.body.position - other.prev_position : splat3(0.0f);
    float t = 0.0f;
    for (uint32_t iteration = 0; iteration < 16u; ++iteration) {
        WorldShape free = sweep_collider(moving, mc, t);
        WorldShape fixed = other_movable ? sweep_collider(other, oc, t)
                                         : world_collider(other.body.position, other.body.orientation, oc);
        ShapeHit gap = pair_gap(w, free, fixed);
        if (gap.distance <= 1e-4f) {  // SWEEP_TOLERANCE, scene.wgsl:1
            if (iteration == 0u && gap.distance <= 0.0f) return none;
            V3 point = free.kind == DYN_SHAPE_PLANE ? free.center : support(w.shapes, free, gap.normal);
            return SweepHit{t, gap.normal, point};
        }
        float closing = dot(free_travel - other_travel, gap.normal) + closing_floor;
        if (closing <= 0.0f) return none;
        t = t + gap.distance / closing;
        if (t >= 1.0f) return none;
    }
    return none;
}

float combine_material(float a, float b, uint32_t mode) {
    if (mode == 1u) return fminw(a, b);
    if (mode == 2u) return fmaxw(a, b);
    if (mode == 3u) return (a + b) * 0.5f;
    return std::sqrt(a * b);
}

// ccd_sweep.wgsl:149-211 over the pairs in sorted order, then ccd_apply.wgsl:7-37 over the dynamic
// rows. The reference keeps the hit that lowers the time first (an atomicMin and a store,
// :158-168), so equal times race on the GPU; here the first pair in (lower, higher collider) order
// keeps it, the rule the library applies.
void ccd(OracleWorld& w) {
    const uint32_t n = (uint32_t)w.states.size();
    std::vector<float> best_time(n, 1.0f);
    std::vector<V4> best_normal(n), best_point(n);
    auto retreat = [&](uint32_t row, const SweepPose& moving, const dyn_collider_record& mc, const SweepPose& other,
                       const dyn_collider_record& oc) {
        SweepHit hit = rigid_sweep(w, moving, mc, other, oc);
        if (!(hit.time < 1.0f) || !(hit.time < best_time[row])) return;
        best_time[row] = hit.time;
        V3 normal = sign_normalize(hit.normal);
        float restitution = combine_material(mc.restitution, oc.restitution, w.params.restitution_combine);
        best_normal[row] = V4{normal.x, normal.y, normal.z, restitution};
        best_point[row] = V4{hit.point.x, hit.point.y, hit.point.z, hit.time};
    };
    for (size_t i = 0; i < w.pair_major.size(); ++i) {
        uint32_t first_slot = w.pair_major[i], second_slot = w.pair_minor[i];
        uint32_t fb = w.owners[first_slot], sb = w.owners[second_slot];
        if (fb == DYN_NO_BODY || sb == DYN_NO_BODY || fb == sb) continue;
        SweepPose first = sweep_body(w, fb), second = sweep_body(w, sb);
        if (!body_moves(first.body) && !body_moves(second.body)) continue;
        const dyn_collider_record& fc = w.colliders[first_slot];
        const dyn_collider_record& sc = w.colliders[second_slot];
        if (fc.kind == DYN_SHAPE_NONE || sc.kind == DYN_SHAPE_NONE) continue;
        uint32_t fg = fc.collision_group != DYN_NO_COLLISION_FILTER ? fc.collision_group : first.body.group;
        uint32_t fm = fc.collision_mask != DYN_NO_COLLISION_FILTER ? fc.collision_mask : first.body.mask;
        uint32_t sg = sc.collision_group != DYN_NO_COLLISION_FILTER ? sc.collision_group : second.body.group;
        uint32_t sm = sc.collision_mask != DYN_NO_COLLISION_FILTER ? sc.collision_mask : second.body.mask;
        if (!((fg & sm) != 0u && (sg & fm) != 0u)) continue;
        if (joined_by_joint(w, fb, sb)) continue;
        retreat(fb, first, fc, second, sc);
        retreat(sb, second, sc, first, fc);
    }
    for (uint32_t row = 0; row < w.params.dynamic_count && row < n; ++row) {
        float time = best_time[row];
        if (!(time < 1.0f)) continue;
        dyn_body_state_record& s = w.states[row];
        const dyn_body_descriptor_record& d = w.descs[row];
        Body b = body_at(w, row);
        V3 axis = xyz(best_normal[row]);
        float restitution = best_normal[row].w;
        V3 lever = xyz(best_point[row]) - body_com(b);
        V3 arm = cross(lever, axis);
        float linear_speed = dot(b.velocity, axis);
        float angular_speed = dot(b.angular_velocity, arm);
        if (linear_speed <= 0.0f && angular_speed <= 0.0f) continue;
        V3 prev_position = rd3(s.prev_position);
        V3 position = prev_position + (b.position - prev_position) * time;
        V4 orientation = quat_slerp(rd4(s.prev_orientation), b.orientation, time);
        V3 velocity = b.velocity, angular = b.angular_velocity;
        if (linear_speed > 0.0f) velocity = velocity - axis * (linear_speed * (1.0f + restitution));
        if (angular_speed > 0.0f) {
            float mass = d.inverse_mass + dot(arm, apply_inverse_inertia_of(d.inverse_inertia, orientation, arm));
            if (mass > 0.0f) {
                float impulse = angular_speed * (1.0f + restitution) / mass;
                velocity = velocity - axis * (impulse * d.inverse_mass);
                angular = angular - apply_inverse_inertia_of(d.inverse_inertia, orientation, arm * impulse);
            }
        }
        wr3(s.position, position);
        wr4(s.orientation, orientation);
        wr3(s.velocity, velocity);
        wr3(s.angular_velocity, angular);
    }
}

// The commit's frozen-contact passes (crates/dynamis-rigid/src/commit.rs:187-208): thaw_contacts.wgsl
// (a frozen contact stays while both bodies were inactive when the step began; one whose body is gone
// is released and its other body disturbed), static_wake_clear.wgsl, freeze_contacts.wgsl (every
// contact whose bodies are both inactive after the step). COUNTER_RESTING is the reference's slot
// count, the most contacts held frozen at once.
void commit_resting(OracleWorld& w) {
    const uint32_t n = (uint32_t)w.states.size();
    std::vector<OracleWorld::Frozen> kept;
    for (const OracleWorld::Frozen& f : w.resting) {
        uint32_t first = resolve_row(w, f.first_id, f.first_generation);
        uint32_t second = resolve_row(w, f.second_id, f.second_generation);
        if (first == DYN_NO_BODY || second == DYN_NO_BODY) {
            if (first != DYN_NO_BODY) w.wake_flags[first] = 1u;
            if (second != DYN_NO_BODY) w.wake_flags[second] = 1u;
            continue;
        }
        if (w.body_activity[first] != 0u || w.body_activity[second] != 0u) continue;
        kept.push_back(f);
    }
    for (uint32_t i = w.params.dynamic_count; i < n; ++i) w.wake_flags[i] = 0u;
    for (const dyn_contact_record& c : w.contacts) {
        uint32_t first = w.owners[c.a], second = w.owners[c.b];
        if (body_is_active(w.states[first], w.descs[first]) || body_is_active(w.states[second], w.descs[second])) continue;
        if (kept.size() >= w.contact_capacity) {
            w.counters[DYN_COUNTER_REFUSED_RESTING] += 1;
            continue;
        }
        kept.push_back(OracleWorld::Frozen{c.first_body_id, c.first_generation, c.second_body_id, c.second_generation, c.a, c.b});
    }
    w.resting.swap(kept);
    w.counters[DYN_COUNTER_RESTING] = std::max(w.counters[DYN_COUNTER_RESTING], (uint32_t)w.resting.size());
}

bool world_has_ccd(const OracleWorld& w) {
    for (const dyn_body_descriptor_record& d : w.descs) {
        if (d.flags & DYN_BODY_CCD) return true;
    }
    return false;
}

void sleep(OracleWorld& w) {
    for (uint32_t i = 0; i < w.params.dynamic_count; ++i) {
        dyn_body_state_record& s = w.states[i];
        if (s.sleeping != 0u || !body_simulates_d(w.descs[i].inverse_mass, w.descs[i].flags)) continue;
        uint32_t root = w.island_parents[i];
        bool disturbed = (w.island_state[root] & DYN_ISLAND_WAKE) != 0u || w.wake_flags[i] != 0u;
        if (disturbed) {
            s.sleep_timer = 0.0f;
        } else {
            s.sleep_timer = s.sleep_timer + w.params.dt;
            if (s.sleep_timer >= w.params.sleep_time) {
                wr3(s.velocity, splat3(0.0f));
                wr3(s.angular_velocity, splat3(0.0f));
                wr3(s.force, splat3(0.0f));
                wr3(s.torque, splat3(0.0f));
                for (int k = 0; k < 3; ++k) s.prev_position[k] = s.position[k];
                for (int k = 0; k < 4; ++k) s.prev_orientation[k] = s.orientation[k];
                s.sleep_timer = 0.0f;
                s.sleeping = 1;
                w.counters[DYN_COUNTER_SLEPT] += 1;
            }
        }
    }
}

}  // namespace

// ---- C API for ctypes (tests and bench only) ----
extern "C" {

OracleWorld* orc_world_create(const dyn_step_params* params, const dyn_body_state_record* states,
                              const dyn_body_descriptor_record* descs, uint32_t n, const dyn_collider_record* colliders,
                              const uint32_t* owners, uint32_t k, const dyn_shape_source_record* sources,
                              uint32_t source_count, const float* vertices, uint32_t vertex_count,
                              uint32_t pair_capacity, uint32_t contact_capacity) {
    for (uint32_t i = 0; i < k; ++i) {
        if (owners[i] != DYN_NO_BODY && owners[i] >= n) return nullptr;  // records that do not fit together
        if (colliders[i].kind == DYN_SHAPE_HULL && colliders[i].source >= source_count) return nullptr;
    }
    OracleWorld* w = new OracleWorld();
    w->params = *params;
    w->params.body_count = n;
    w->params.collider_count = k;
    w->states.assign(states, states + n);
    w->descs.assign(descs, descs + n);
    w->colliders.assign(colliders, colliders + k);
    w->owners.assign(owners, owners + k);
    w->sources.assign(sources, sources + source_count);
    w->vertices.resize(vertex_count);
    for (uint32_t i = 0; i < vertex_count; ++i) {
        w->vertices[i] = V4{vertices[4 * i], vertices[4 * i + 1], vertices[4 * i + 2], vertices[4 * i + 3]};
    }
    w->shapes.sources = w->sources.data();
    w->shapes.source_count = source_count;
    w->shapes.vertices = w->vertices.data();
    w->shapes.vertex_count = vertex_count;
    uint32_t max_id = 0;
    for (uint32_t i = 0; i < n; ++i) max_id = std::max(max_id, states[i].body_id + 1);
    w->row_of_id.assign(max_id, DYN_NO_BODY);
    for (uint32_t i = 0; i < n; ++i) w->row_of_id[states[i].body_id] = i;
    w->pair_capacity = pair_capacity;
    w->contact_capacity = contact_capacity;
    w->wake_flags.assign(n, 0);
    return w;
}

void orc_world_destroy(OracleWorld* w) { delete w; }

// Constraints in row order with their body rows and runtime records; plans the solve order.
// Returns 0 when a row is out of range or a kind other than the ball joint appears.
uint32_t orc_set_constraints(OracleWorld* w, const dyn_constraint_descriptor_record* descs,
                             const dyn_constraint_rows_record* rows, const dyn_constraint_runtime_record* runtime,
                             uint32_t m) {
    uint32_t n = (uint32_t)w->states.size();
    for (uint32_t j = 0; j < m; ++j) {
        if (rows[j].first_row >= n || rows[j].second_row >= n || descs[j].kind != DYN_CONSTRAINT_BALL) return 0;
    }
    w->joint_descs.assign(descs, descs + m);
    w->joint_rows.assign(rows, rows + m);
    w->joint_runtime.assign(runtime, runtime + m);
    plan_joint_order(*w);
    w->params.constraint_count = m;
    return 1;
}

// Queues body commands for the next step by row (the caller maps body ids to rows).
void orc_queue_edits(OracleWorld* w, const uint32_t* rows, const dyn_body_edit_record* edits, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) w->edits.emplace_back(rows[i], edits[i]);
}

void orc_set_body_worlds(OracleWorld* w, const uint32_t* rows, uint32_t n) {
    w->body_world.assign(rows, rows + n);
    w->held_run.clear();  // the library uploads the scene again, which keeps no grid run
    w->held_base = 0;
}

uint32_t orc_constraints(const OracleWorld* w, dyn_constraint_runtime_record* out) {
    if (out) std::memcpy(out, w->joint_runtime.data(), w->joint_runtime.size() * sizeof(*out));
    return (uint32_t)w->joint_runtime.size();
}

void orc_joint_plan(const OracleWorld* w, uint32_t* rows, uint32_t* layers, uint32_t* components, uint32_t* sizes) {
    if (rows) std::memcpy(rows, w->plan_rows.data(), w->plan_rows.size() * 4);
    if (layers) std::memcpy(layers, w->plan_layers.data(), w->plan_layers.size() * 4);
    if (components) std::memcpy(components, w->plan_components.data(), w->plan_components.size() * 4);
    if (sizes) {
        sizes[0] = (uint32_t)w->plan_rows.size();
        sizes[1] = (uint32_t)(w->plan_layers.size() / 2);
        sizes[2] = (uint32_t)(w->plan_components.size() / 2);
    }
}

void orc_step(OracleWorld* w, float dt) {
    w->params.dt = dt;
    w->params.substep_dt = dt / (float)w->params.substeps;
    apply_commands(*w);
    prepare(*w);
    emit_entries(*w);
    broadphase(*w);
    narrowphase(*w);
    build_islands(*w);
    wake_and_live(*w);
    solver_prepare(*w);
    w->solve_contacts = w->contacts;
    solve_substeps(*w);
    if (world_has_ccd(*w)) ccd(*w);
    sleep(*w);
    commit_resting(*w);
    w->archive = w->contacts;  // commit: contact_archive.wgsl + archive_count_sync.wgsl
    w->counters[DYN_COUNTER_ARCHIVED] = (uint32_t)w->archive.size();
    w->counters[DYN_COUNTER_STEP] += 1;
}

void orc_counters(const OracleWorld* w, uint32_t* out) {
    for (uint32_t i = 0; i < DYN_COUNTER_DEVICE_COUNT; ++i) out[i] = w->counters[i];
}
uint32_t orc_states(const OracleWorld* w, dyn_body_state_record* out) {
    if (out) std::memcpy(out, w->states.data(), w->states.size() * sizeof(dyn_body_state_record));
    return (uint32_t)w->states.size();
}
uint32_t orc_aabbs(const OracleWorld* w, float* out) {
    if (out) {
        for (size_t i = 0; i < w->aabbs.size(); ++i) {
            wr3(out + 8 * i, w->aabbs[i].min);
            out[8 * i + 3] = 0.0f;
            wr3(out + 8 * i + 4, w->aabbs[i].max);
            out[8 * i + 7] = 0.0f;
        }
    }
    return (uint32_t)w->aabbs.size();
}
uint32_t orc_entry_keys(const OracleWorld* w, uint32_t* keys, uint32_t* colliders) {
    size_t e = w->entry_keys.size();
    for (size_t i = 0; i < e && keys; ++i) {
        keys[i] = w->entry_keys[i];
        colliders[i] = w->entries[w->entry_order[i]].info;
    }
    return (uint32_t)e;
}
uint32_t orc_pairs(const OracleWorld* w, uint32_t* major, uint32_t* minor) {
    size_t p = w->pair_major.size();
    if (major) {
        std::memcpy(major, w->pair_major.data(), p * 4);
        std::memcpy(minor, w->pair_minor.data(), p * 4);
    }
    return (uint32_t)p;
}
uint32_t orc_contacts(const OracleWorld* w, dyn_contact_record* out) {
    if (out) std::memcpy(out, w->contacts.data(), w->contacts.size() * sizeof(dyn_contact_record));
    return (uint32_t)w->contacts.size();
}
// The last step's frozen contact set: the contacts as its substeps received them (accumulated
// impulses after the relay), their target speeds (4 per contact) and relay sources (4 per contact:
// 4 x archived contact + archived point, -1 when not relayed). Returns the contact count.
uint32_t orc_solve_contacts(const OracleWorld* w, dyn_contact_record* out, float* targets, int32_t* sources) {
    const size_t c = w->solve_contacts.size();
    if (out) std::copy(w->solve_contacts.begin(), w->solve_contacts.end(), out);
    if (targets) std::copy(w->target_speeds.begin(), w->target_speeds.begin() + 4 * c, targets);
    if (sources) std::copy(w->relay_source.begin(), w->relay_source.begin() + 4 * c, sources);
    return (uint32_t)c;
}
// Keeps (or stops keeping) the primal snapshots of each step (OracleWorld::snap_pose ...).
void orc_keep_snapshots(OracleWorld* w, uint32_t keep) { w->keep_snapshots = keep != 0u; }
void orc_set_solver_guard(OracleWorld* w, uint32_t flags) { w->solver_guard = flags; }
// World::set_ccd on a row's descriptor (the library's dyn_set_ccd); the caller queues the wake.
void orc_set_ccd(OracleWorld* w, uint32_t row, uint32_t enabled) {
    if (row >= w->descs.size()) return;
    if (enabled) {
        w->descs[row].flags |= DYN_BODY_CCD;
    } else {
        w->descs[row].flags &= ~DYN_BODY_CCD;
    }
}
void orc_step_snapshots(const OracleWorld* w, float* pose, float* vel, float* acc, float* res) {
    if (pose) std::copy(w->snap_pose.begin(), w->snap_pose.end(), pose);
    if (vel) std::copy(w->snap_vel.begin(), w->snap_vel.end(), vel);
    if (acc) std::copy(w->snap_acc.begin(), w->snap_acc.end(), acc);
    if (res) std::copy(w->snap_res.begin(), w->snap_res.end(), res);
}
// The last step's branch decisions (OracleWorld::solve_flags ...); any output may be null.
void orc_step_decisions(const OracleWorld* w, uint8_t* solve, uint8_t* position, uint8_t* integrate, uint8_t* targets) {
    if (solve) std::copy(w->solve_flags.begin(), w->solve_flags.end(), solve);
    if (position) std::copy(w->position_flags.begin(), w->position_flags.end(), position);
    if (integrate) std::copy(w->integrate_flags.begin(), w->integrate_flags.end(), integrate);
    if (targets) std::copy(w->target_flags.begin(), w->target_flags.end(), targets);
}
// The frozen contacts, six words each (first id, its generation, second id, its generation,
// collider a, collider b), in the order they were frozen.
uint32_t orc_resting(const OracleWorld* w, uint32_t* out) {
    if (out) {
        for (size_t i = 0; i < w->resting.size(); ++i) {
            const OracleWorld::Frozen& f = w->resting[i];
            const uint32_t row[6] = {f.first_id, f.first_generation, f.second_id, f.second_generation, f.a, f.b};
            std::memcpy(out + 6 * i, row, sizeof(row));
        }
    }
    return (uint32_t)w->resting.size();
}

uint32_t orc_islands(const OracleWorld* w, uint32_t* out) {
    if (out) std::memcpy(out, w->island_parents.data(), w->island_parents.size() * 4);
    return (uint32_t)w->island_parents.size();
}

// Known-answer hooks for the math and sort restatements.
// Host threads for the parallel loops (results do not depend on the count).
uint32_t orc_threads(void) {
#ifdef _OPENMP
    return (uint32_t)omp_get_max_threads();
#else
    return 1u;
#endif
}
void orc_set_threads(uint32_t n) {
#ifdef _OPENMP
    omp_set_num_threads((int)std::max(n, 1u));
#else
    (void)n;
#endif
}

float orc_sin(float x) { return osin(x); }
float orc_cos(float x) { return ocos(x); }
float orc_atan2(float y, float x) { return oatan2(y, x); }
uint32_t orc_key_words(uint32_t n) { return key_words(n); }
void orc_radix_sort(uint32_t* major, uint32_t* minor, uint32_t* payload, uint32_t n, uint32_t major_words,
                    uint32_t minor_words) {
    std::vector<uint32_t> a(major, major + n), b(minor, minor + n), c;
    if (payload) c.assign(payload, payload + n);
    radix_sort_pairs(a, b, payload ? &c : nullptr, major_words, minor_words);
    std::memcpy(major, a.data(), n * 4);
    std::memcpy(minor, b.data(), n * 4);
    if (payload) std::memcpy(payload, c.data(), n * 4);
}

// The triangles of hull source `source` (index triples), for the scene queries' hull tests.
void orc_set_hull_triangles(OracleWorld* w, uint32_t source, const uint32_t* tris, uint32_t n) {
    if (w->hull_tri_ranges.size() < 2 * ((size_t)source + 1)) w->hull_tri_ranges.resize(2 * ((size_t)source + 1), 0u);
    w->hull_tri_ranges[2 * (size_t)source] = (uint32_t)(w->hull_tris.size() / 3);
    w->hull_tri_ranges[2 * (size_t)source + 1] = n;
    w->hull_tris.insert(w->hull_tris.end(), tris, tris + 3 * (size_t)n);
}

// query_world_aabb (scene_cast.wgsl:341-362)
Aabb query_world_box(const OracleWorld& w, const dyn_query_record& q) {
    V3 origin = q_origin(q);
    if (q.kind == DYN_QUERY_RAY) {
        V3 end = origin + normalize(q_direction(q)) * q.extent;
        return Aabb{vmin(origin, end), vmax(origin, end)};
    }
    if (q.kind == DYN_QUERY_SWEEP) {
        Aabb a = world_aabb_of(w.shapes, query_shape(q, origin));
        Aabb b = world_aabb_of(w.shapes, query_shape(q, origin + normalize(q_direction(q)) * q.extent));
        return Aabb{vmin(a.min, b.min), vmax(a.max, b.max)};
    }
    return world_aabb_of(w.shapes, query_shape(q, origin));
}

// The candidates of one query (grid_index.wgsl:289-388, scene_cast.wgsl:90-134): the colliders with
// an entry in a cell the query's box covers, level by level; a level under which the box covers
// more than GRID_WALK_CELLS cells is taken whole, its entries tested against the box. `grid` is the
// world's index rebuilt from its current states. Sets *spilled when more than QUERY_CANDIDATES
// entries were gathered (the reference then keeps whichever landed first; here all are kept).
std::vector<uint32_t> query_candidates(const OracleWorld& grid, const Aabb& box, bool* spilled) {
    std::vector<uint32_t> out;
    const float base = grid_base_cell(grid);
    uint32_t occupied = grid.counters[DYN_COUNTER_GRID_LEVELS] | grid.counters[DYN_COUNTER_RESTING_LEVELS] |
                        grid.counters[DYN_COUNTER_IMMOVABLE_LEVELS];
    const std::vector<uint32_t>& keys = grid.entry_keys;
    while (occupied != 0u) {
        const uint32_t level = (uint32_t)__builtin_ctz(occupied);
        occupied &= occupied - 1u;
        const float cs = level_cell_size(level, base);
        const I3 lo = floor_div(box.min, cs), hi = floor_div(box.max, cs);
        const int64_t sx = (int64_t)hi.x - lo.x + 1, sy = (int64_t)hi.y - lo.y + 1, sz = (int64_t)hi.z - lo.z + 1;
        const int64_t cells = sx * sy * sz;
        if (cells <= 0) continue;
        if (cells > 4096) {
            auto first = std::lower_bound(keys.begin(), keys.end(), level << DYN_LEVEL_KEY_SHIFT);
            auto end = std::lower_bound(keys.begin(), keys.end(), (level + 1u) << DYN_LEVEL_KEY_SHIFT);
            for (auto it = first; it != end; ++it) {
                const Entry& e = grid.entries[grid.entry_order[it - keys.begin()]];
                if (aabb_overlaps(e.box, box)) out.push_back(e.info & DYN_ENTRY_INDEX_MASK);
            }
        } else {
            for (int x = lo.x; x <= hi.x; ++x)
                for (int y = lo.y; y <= hi.y; ++y)
                    for (int z = lo.z; z <= hi.z; ++z) {
                        const uint32_t key = cell_key_in(level, I3{x, y, z}, 0u);
                        auto it = std::lower_bound(keys.begin(), keys.end(), key);
                        for (; it != keys.end() && *it == key; ++it)
                            out.push_back(grid.entries[grid.entry_order[it - keys.begin()]].info & DYN_ENTRY_INDEX_MASK);
                    }
        }
    }
    *spilled = out.size() > DYN_QUERY_CANDIDATES;
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
    return out;
}

// A batch of scene queries against the world's current states (scene_cast.wgsl:434-533): the grid
// index is rebuilt from the current states on a copy of the world (the AABB and entry passes of a
// step, as the reference's query run and dyn_query rebuild it), each query's candidates are walked
// from it, the hits are ordered by (distance key, collider slot) and at most
// min(max_hits, QUERY_CANDIDATES) are written from hit_base; count and overflow are set. hit_base is
// assigned in submission order, as World::submit_query does.
void orc_query(const OracleWorld* cw, dyn_query_record* queries, uint32_t n, dyn_query_hit_record* hits) {
    const OracleWorld& w = *cw;
    OracleWorld grid = w;
    for (uint32_t c : {DYN_COUNTER_GRID_LEVELS, DYN_COUNTER_IMMOVABLE_LEVELS, DYN_COUNTER_RESTING_LEVELS,
                       DYN_COUNTER_GRID_SCALE, DYN_COUNTER_GRID_EXTENT, DYN_COUNTER_ENTRIES, DYN_COUNTER_IMMOVABLE_ENTRIES,
                       DYN_COUNTER_RESTING_ENTRIES, DYN_COUNTER_IMMOVABLE_EMITTED, DYN_COUNTER_COARSE_ACTIVE,
                       DYN_COUNTER_ENTRY_FAULTS})
        grid.counters[c] = 0u;
    grid.body_activity.resize(grid.states.size(), 0u);
    grid.wake_flags.resize(grid.states.size(), 0u);
    prepare(grid);
    emit_entries(grid);
    HullTriangles ht{w.hull_tris.data(), w.hull_tri_ranges.data(), (uint32_t)(w.hull_tri_ranges.size() / 2)};
    uint32_t base = 0;
    for (uint32_t qi = 0; qi < n; ++qi) {
        dyn_query_record& q = queries[qi];
        q.hit_base = base;
        const uint32_t capacity = std::min(q.max_hits, DYN_QUERY_CANDIDATES);
        base += capacity;
        struct Found {
            uint64_t key;
            ShapeHit hit;
            uint32_t slot;
        };
        std::vector<Found> found;
        const bool colliders = (q.filters.targets & DYN_QUERY_TARGET_COLLIDERS) != 0u;
        bool spilled = false;
        const std::vector<uint32_t> candidates =
            colliders ? query_candidates(grid, query_world_box(w, q), &spilled) : std::vector<uint32_t>();
        for (uint32_t slot : candidates) {
            const uint32_t row = w.owners[slot];
            if (row == DYN_NO_BODY) continue;
            const dyn_body_state_record& st = w.states[row];
            const dyn_body_descriptor_record& d = w.descs[row];
            const dyn_collider_record& c = w.colliders[slot];
            const dyn_query_filter_record& f = q.filters;
            if (f.exclude_id != DYN_NO_BODY && st.body_id == f.exclude_id && st.generation == f.exclude_generation) continue;
            if (f.include_id != DYN_NO_BODY && (st.body_id != f.include_id || st.generation != f.include_generation)) continue;
            if ((f.flags & DYN_FILTER_IGNORE_SENSORS) && (c.flags & DYN_COLLIDER_SENSOR)) continue;
            if ((f.flags & DYN_FILTER_IGNORE_SLEEPING) && st.sleeping != 0u) continue;
            if ((f.flags & DYN_FILTER_IGNORE_STATIC) && !body_moves_d(d.inverse_mass, d.flags)) continue;
            if ((f.flags & DYN_FILTER_IGNORE_KINEMATIC) && body_moves_d(d.inverse_mass, d.flags) &&
                !body_simulates_d(d.inverse_mass, d.flags))
                continue;
            if (f.group != 0u) {
                uint32_t group = c.collision_group != DYN_NO_COLLISION_FILTER ? c.collision_group : d.collision_group;
                uint32_t mask = c.collision_mask != DYN_NO_COLLISION_FILTER ? c.collision_mask : d.collision_mask;
                if (!((f.group & mask) != 0u && (group & f.mask) != 0u)) continue;
            }
            if (c.kind == DYN_SHAPE_NONE) continue;
            WorldShape world = world_collider(rd3(st.position), rd4(st.orientation), c);
            ShapeHit hit = resolve_hit(w.shapes, ht, q, world);
            if (!(hit.distance < kNoHit)) continue;
            found.push_back(Found{((uint64_t)hit_key(hit.distance) << 32) | slot, hit, slot});
        }
        std::sort(found.begin(), found.end(), [](const Found& a, const Found& b) { return a.key < b.key; });
        const uint32_t emitted = std::min<uint32_t>(capacity, (uint32_t)found.size());
        for (uint32_t i = 0; i < emitted; ++i) {
            const Found& h = found[i];
            const dyn_body_state_record& st = w.states[w.owners[h.slot]];
            dyn_query_hit_record r{};
            r.body_id = st.body_id;
            r.body_generation = st.generation;
            r.distance = h.hit.distance;
            r.scene_target = (DYN_ENTRY_KIND_COLLIDER << DYN_ENTRY_KIND_SHIFT) | h.slot;
            wr3(r.point, h.hit.point);
            r.triangle = h.hit.triangle;
            wr3(r.normal, h.hit.normal);
            r.surface = DYN_NO_SURFACE;
            hits[q.hit_base + i] = r;
        }
        q.count = emitted;
        q.overflow = (spilled || emitted < found.size()) ? 1u : 0u;
    }
}

// One pair through the narrowphase restatement (bodies/colliders from the world).
uint32_t orc_narrowphase_pair(const OracleWorld* w, uint32_t a, uint32_t b, dyn_contact_record* out) {
    return narrowphase_pair(*w, a, b, out) ? 1u : 0u;
}

}  // extern "C"
