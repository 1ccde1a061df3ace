// step.cuh - the sm_100a kernels of one rigid-body step.
//
// One kernel per stage of World::step (crates/dynamis-rigid/src/lib.rs:119-153); each cites the
// WGSL pass it replaces. Counts produced on the device (entries, pairs, contacts, live rows,
// solver rows) stay on the device in the control words; kernels grid-stride over them, so the
// whole step is replayed as one CUDA graph with no host round trip. Appends use coalesced-group
// aggregated atomics; every order that depends on those atomics (pair emission, live list,
// solver rows, staging slots) is either sorted afterwards or irrelevant to the result.
#pragma once

#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include "dmath.cuh"
#include "layout.cuh"
#include "narrow.cuh"
#include "sort.cuh"

namespace dyn {

namespace cg = cooperative_groups;

// Aggregated append: every lane of the calling coalesced group must pass the same counter.
__device__ __forceinline__ uint32_t append_slot(uint32_t* counter) {
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(counter, g.size());
    return g.shfl(base, 0) + g.thread_rank();
}
__device__ __forceinline__ void add_counter(uint32_t* counter, uint32_t value) {
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t total = cg::reduce(g, value, cg::plus<uint32_t>());
    if (g.thread_rank() == 0 && total) atomicAdd(counter, total);
}
__device__ __forceinline__ void max_counter(uint32_t* counter, uint32_t value) {
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t m = cg::reduce(g, value, cg::greater<uint32_t>());
    if (g.thread_rank() == 0) atomicMax(counter, m);
}
__device__ __forceinline__ void or_counter(uint32_t* counter, uint32_t value) {
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t m = cg::reduce(g, value, cg::bit_or<uint32_t>());
    if (g.thread_rank() == 0 && m) atomicOr(counter, m);
}

#define GRID_STRIDE(i, n) for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

// Counters that persist across steps (crates/dynamis-abi/src/counter.rs: Maintained).
__global__ void k_reset(DeviceWorld w) {
    for (uint32_t i = threadIdx.x; i < DYN_COUNTER_DEVICE_COUNT; i += blockDim.x) {
        if (i == DYN_COUNTER_ARCHIVED || i == DYN_COUNTER_STEP || i == DYN_COUNTER_RESTING) continue;
        w.counters[i] = 0u;
    }
    if (threadIdx.x == 0) w.held[HELD_STALE] = 0u;
    for (uint32_t i = threadIdx.x; i < CTL_COUNT; i += blockDim.x) {
        if (i == CTL_ARCHIVED || i == CTL_STATUS || i == CTL_RESTING) continue;
        w.ctl[i] = 0u;
    }
}

// clear_inputs.wgsl, activity.wgsl (all rows); begin_step.wgsl, island_init.wgsl (dynamic rows);
// solver_reset.wgsl (all rows). Folding them into one pass changes nothing: none of them reads
// what another writes.
// clear_inputs.wgsl on its own, for steps that apply body edits between it and the rest.
__global__ void k_clear_inputs(DeviceWorld w) {
    GRID_STRIDE(i, w.n) {
        w.force[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        w.torque[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

// body_edits.wgsl: the queued commands of one body row, in order, after the inputs are cleared and
// before anything reads the rows.
__device__ __forceinline__ void edit_disturbs(const DeviceWorld& w, uint32_t row, uint32_t* sleeping, float* timer, bool disturbed) {
    if (*sleeping != 0u) {
        atomicAdd(&w.counters[DYN_COUNTER_WOKE], 1u);
        atomicOr(&w.wake_flags[row], 1u);
    } else if (disturbed) {
        atomicOr(&w.wake_flags[row], 1u);
    }
    *sleeping = 0u;
    *timer = 0.0f;
}
__global__ void k_body_edits(DeviceWorld w) {
    const uint32_t runs = *w.edit_count;
    GRID_STRIDE(r, runs) {
        const uint4 run = w.edit_runs[r];
        const uint32_t row = run.x;
        if (row >= w.n || run.z == 0u) continue;
        BodyHot& h = w.hot[row];
        f3 position = xyz(h.pos), velocity = xyz(h.vel), angular = xyz(h.ang);
        float4 orientation = h.rot;
        f3 prev_position = xyz(w.prev_pos[row]);
        float4 prev_orientation = w.prev_rot[row];
        f3 force = xyz(w.force[row]), torque = xyz(w.torque[row]);
        uint32_t sleeping = h.aux.x;
        float timer = w.sleep_timer[row];
        const float im = h.pos.w;
        const uint32_t flags = h.aux.y;
        const f3 com_local = xyz(h.com);
        const float4 ii0 = h.ii0;
        const float2 ii1 = make_float2(h.ii1.x, h.ii1.y);
        for (uint32_t k = 0; k < run.z; ++k) {
            const dyn_body_edit_record& e = w.edits[run.y + k];
            const f3 ev = mk3(e.state.velocity[0], e.state.velocity[1], e.state.velocity[2]);
            const f3 ep = mk3(e.state.position[0], e.state.position[1], e.state.position[2]);
            if (e.kind == DYN_EDIT_PATCH) {
                if (e.mask & DYN_PATCH_POSITION) {
                    position = ep;
                    prev_position = ep;
                }
                if (e.mask & DYN_PATCH_ORIENTATION) {
                    orientation = make_float4(e.state.orientation[0], e.state.orientation[1], e.state.orientation[2],
                                              e.state.orientation[3]);
                    prev_orientation = orientation;
                }
                if (e.mask & DYN_PATCH_VELOCITY) velocity = ev;
                if (e.mask & DYN_PATCH_ANGULAR_VELOCITY)
                    angular = mk3(e.state.angular_velocity[0], e.state.angular_velocity[1], e.state.angular_velocity[2]);
                const bool teleport = (e.mask & (DYN_PATCH_POSITION | DYN_PATCH_ORIENTATION)) != 0u;
                edit_disturbs(w, row, &sleeping, &timer, teleport || !simulates(im, flags));
            } else if (e.kind == DYN_EDIT_FORCE) {
                force = force + mk3(e.state.force[0], e.state.force[1], e.state.force[2]);
                edit_disturbs(w, row, &sleeping, &timer, false);
            } else if (e.kind == DYN_EDIT_FORCE_AT_POINT) {
                const f3 f = mk3(e.state.force[0], e.state.force[1], e.state.force[2]);
                force = force + f;
                torque = torque + cross(ep - (position + quat_rotate(orientation, com_local)), f);
                edit_disturbs(w, row, &sleeping, &timer, false);
            } else if (e.kind == DYN_EDIT_TORQUE) {
                torque = torque + mk3(e.state.torque[0], e.state.torque[1], e.state.torque[2]);
                edit_disturbs(w, row, &sleeping, &timer, false);
            } else if (e.kind == DYN_EDIT_IMPULSE) {
                velocity = velocity + ev * im;
                edit_disturbs(w, row, &sleeping, &timer, false);
            } else if (e.kind == DYN_EDIT_IMPULSE_AT_POINT) {
                velocity = velocity + ev * im;
                const f3 lever = ep - (position + quat_rotate(orientation, com_local));
                angular = angular + inv_inertia_world(ii0, ii1, orientation, cross(lever, ev));
                edit_disturbs(w, row, &sleeping, &timer, false);
            } else if (e.kind == DYN_EDIT_ANGULAR_IMPULSE) {
                angular = angular + inv_inertia_world(ii0, ii1, orientation,
                                                      mk3(e.state.angular_velocity[0], e.state.angular_velocity[1],
                                                          e.state.angular_velocity[2]));
                edit_disturbs(w, row, &sleeping, &timer, false);
            } else if (e.kind == DYN_EDIT_SLEEP) {
                if (sleeping == 0u) atomicAdd(&w.counters[DYN_COUNTER_SLEPT], 1u);
                velocity = s3(0.0f);  // freeze_body (core.wgsl:218-227)
                angular = s3(0.0f);
                force = s3(0.0f);
                torque = s3(0.0f);
                prev_position = position;
                prev_orientation = orientation;
                timer = 0.0f;
                sleeping = 1u;
                atomicExch(&w.wake_flags[row], 0u);
            } else if (e.kind == DYN_EDIT_WAKE) {
                if (sleeping != 0u) atomicAdd(&w.counters[DYN_COUNTER_WOKE], 1u);
                timer = 0.0f;
                sleeping = 0u;
                atomicOr(&w.wake_flags[row], 1u);
            }
        }
        h.pos = mk4(position, im);
        h.rot = orientation;
        h.vel = mk4(velocity, 0.0f);
        h.ang = mk4(angular, 0.0f);
        h.aux.x = sleeping;
        w.prev_pos[row] = mk4(prev_position, 0.0f);
        w.prev_rot[row] = prev_orientation;
        w.force[row] = mk4(force, 0.0f);
        w.torque[row] = mk4(torque, 0.0f);
        w.sleep_timer[row] = timer;
    }
}

template <bool kClearInputs>
__global__ void k_begin(DeviceWorld w, dyn_step_params p) {
    GRID_STRIDE(i, w.n) {
        if (kClearInputs) {
            w.force[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            w.torque[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        BodyHot& h = w.hot[i];
        float im = h.pos.w;
        uint32_t flags = h.aux.y;
        uint32_t sleeping = h.aux.x;
        bool mv = moves(im, flags);
        bool sim = simulates(im, flags);
        bool awake = mv && sleeping == 0u;
        w.activity[i] = awake ? 1u : 0u;
        f3 v = xyz(h.vel), av = xyz(h.ang);
        bool moving;
        if (mv && !sim && (!is_zero3(v) || !is_zero3(av))) {
            moving = true;
        } else if (!sim || sleeping != 0u) {
            moving = false;
        } else {
            float2 th = w.thresh[i];
            float sv = (flags & DYN_OVERRIDE_SLEEP_LINEAR) ? th.x : p.sleep_velocity;
            float sw = (flags & DYN_OVERRIDE_SLEEP_ANGULAR) ? th.y : p.sleep_angular_velocity;
            moving = length(v) > sv || length(av) > sw;
        }
        w.motion[i] = moving ? 1u : 0u;
        if (awake) w.counters[DYN_COUNTER_ACTIVE] = 1u;
        if (i < w.nd) {
            if (sleeping == 0u) {
                w.prev_pos[i] = make_float4(h.pos.x, h.pos.y, h.pos.z, 0.0f);
                w.prev_rot[i] = h.rot;
            }
            w.parents[i] = i;
            w.istate[i] = 0u;
        }
        h.aux.z = 0u;
        w.row_flag[i] = 0u;
        w.resolution[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

__device__ __forceinline__ float grid_extent_of(f3 mn, f3 mx) { return wmax(wmax(mx.x - mn.x, mx.y - mn.y), mx.z - mn.z); }

// broadphase_aabb.wgsl:11-62 (core.wgsl:109-126 for the grid resolution)
__global__ void k_aabb(DeviceWorld w, dyn_step_params p) {
    GRID_STRIDE(i, w.k) {
        uint32_t owner = w.c_owner[i];
        if (owner == DYN_NO_BODY) {
            w.c_class[i] = make_uint4(DYN_NO_BODY, 0u, 0u, 0u);
            continue;
        }
        DBody b = load_dbody(w.hot, owner);
        DColl c = load_dcoll(w, i);
        {  // what k_pair_class asks of this collider, in one record (nothing it reads changes before it runs)
            const uint4 id = w.ident[owner];
            const uint2 f = w.c_filter[i];
            const bool unscaled = veq(c.scale, s3(1.0f));
            w.c_class[i] = make_uint4(owner, f.x != DYN_NO_COLLISION_FILTER ? f.x : id.z,
                                      f.y != DYN_NO_COLLISION_FILTER ? f.y : id.w,
                                      c.kind | (moves(b.inverse_mass, b.flags) ? 0x100u : 0u) | (unscaled ? 0x200u : 0u));
        }
        WShape s = world_shape(b.position, b.orientation, c);
        DAabb tight = world_aabb(w, s);
        WShape up = s;
        up.rotation = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        DAabb res = world_aabb(w, up);
        float extent = grid_extent_of(res.min, res.max);
        float scale = extent <= 0.0f ? 0.0f : wclamp(1.0f / extent, 1.0f / 1e12f, 1e12f);
        max_counter(&w.counters[DYN_COUNTER_GRID_SCALE], fbits(scale));
        max_counter(&w.counters[DYN_COUNTER_GRID_EXTENT], fbits(wmax(extent, 0.0f)));
        DAabb swept = tight;
        if (moves(b.inverse_mass, b.flags)) {
            f3 travel = vabs(b.velocity * p.dt);
            float spin = length(b.angular_velocity * p.dt);
            f3 center = b.position + quat_rotate(b.orientation, c.offset);
            float radius = length((tight.max - tight.min) * 0.5f) + length(center - dbody_com(b));
            float rr = spin >= 3.141592653589793f ? 2.0f * radius : 2.0f * radius * dsin(0.5f * spin);
            f3 reach = s3(p.contact_margin + rr);
            swept.min = tight.min - travel - reach;
            swept.max = tight.max + travel + reach;
        }
        w.aabb[2 * i] = mk4(swept.min, 0.0f);
        w.aabb[2 * i + 1] = mk4(swept.max, 0.0f);
    }
}

// ---- grid (grid_index.wgsl:28-287) ----
struct I3 {
    int x, y, z;
};
__device__ __forceinline__ float base_cell(const DeviceWorld& w) {
    float scale = bitsf(w.counters[DYN_COUNTER_GRID_SCALE]);
    float extent = bitsf(w.counters[DYN_COUNTER_GRID_EXTENT]);
    float finest = scale > 0.0f ? 1.0f / scale : 1e12f;
    return wmax(finest, extent * 9.31322574615478515625e-10f);
}
__device__ __forceinline__ I3 floor_div(f3 v, float cs) {
    return I3{(int)floorf(v.x / cs), (int)floorf(v.y / cs), (int)floorf(v.z / cs)};
}
__device__ __forceinline__ float level_size(uint32_t level, float cs) { return cs * (float)(1u << level); }
__device__ __forceinline__ uint32_t cell_hash(I3 c) {
    uint32_t x = (uint32_t)c.x * 0x9E3779B9u;
    uint32_t y = (uint32_t)c.y * 0x85EBCA77u;
    uint32_t z = (uint32_t)c.z * 0xC2B2AE3Du;
    return (x ^ y ^ z ^ (x << 7) ^ (y >> 3) ^ (z << 11)) & DYN_CELL_HASH_MASK;
}
__device__ __forceinline__ uint32_t cell_key(uint32_t level, I3 c) { return (level << DYN_LEVEL_KEY_SHIFT) | cell_hash(c); }
// Batched worlds: the sub-world of a row is mixed into its cells' hash, so the grids of different
// sub-worlds share no cell (up to hash collisions, which the pair test rejects). World 0 mixes in
// nothing, so a single world's keys are the reference's. The odd multiplier keeps distinct worlds
// distinct modulo the 27-bit hash.
__device__ __forceinline__ uint32_t world_mix(uint32_t world) { return world * 0x2545F491u; }
__device__ __forceinline__ uint32_t cell_key_in(uint32_t level, I3 c, uint32_t world) {
    return (level << DYN_LEVEL_KEY_SHIFT) | ((cell_hash(c) ^ world_mix(world)) & DYN_CELL_HASH_MASK);
}
__device__ __forceinline__ uint32_t shape_levels(f3 mn, f3 mx, float base) {
    uint32_t level = 0;
    for (;;) {
        float cs = level_size(level, base);
        I3 a = floor_div(mn, cs), b = floor_div(mx, cs);
        uint32_t sx = (uint32_t)(b.x - a.x + 1), sy = (uint32_t)(b.y - a.y + 1), sz = (uint32_t)(b.z - a.z + 1);
        uint32_t m = max(max(sx, sy), sz);
        if (m <= DYN_MAX_CELLS_PER_AXIS || level >= DYN_GRID_LEVEL_LIMIT) break;
        level += 1;
    }
    return level;
}

// The run a live collider's entries belong to this step (grid_resting_entries.wgsl:11-19: a
// movable body that is not active goes to the resting run; immovable_entries.wgsl: a body that does
// not move to the immovable run).
__device__ __forceinline__ uint32_t grid_run(bool mv, bool awake) {
    return !mv ? RUN_IMMOVABLE : (awake ? RUN_AWAKE : RUN_RESTING);
}
// The info word of collider i's entry at cell offset `offset` (collider_emit.wgsl:31-63).
__device__ __forceinline__ uint32_t entry_info(uint32_t i, uint32_t offset, bool mv, bool awake) {
    uint32_t info = i | (offset << DYN_ENTRY_CELL_SHIFT) | (DYN_ENTRY_KIND_COLLIDER << DYN_ENTRY_KIND_SHIFT);
    if (mv && awake) info |= DYN_ENTRY_AWAKE;
    if (mv) info |= DYN_ENTRY_MOBILE;
    if (offset == 0u) info |= DYN_ENTRY_PRIMARY;
    return info;
}
__device__ __forceinline__ bool same_bits(f3 a, float4 b) {
    return __float_as_uint(a.x) == __float_as_uint(b.x) && __float_as_uint(a.y) == __float_as_uint(b.y) &&
           __float_as_uint(a.z) == __float_as_uint(b.z);
}

// collider_emit.wgsl:6-29 (level, cell budget) for every collider, and the counters of the three
// runs. A step (kStep) also sorts each collider into its run and checks that a kept run still holds
// the entries its members would emit now: the same members, each with the box, owner and info its
// first slot holds (the rest of its slots follow from them at an unchanged resolution, which the
// gate checks). A collider that left a kept run, joined one, or whose box moved marks that run
// stale. A query (not kStep) counts every collider's entries for one compact scan.
template <bool kStep>
__global__ void k_entry_count(DeviceWorld w) {
    float base = base_cell(w);
    uint32_t stale = 0u;
    GRID_STRIDE(i, w.k) {
        uint32_t owner = w.c_owner[i];
        uint32_t emitted = 0, run = RUN_NONE;
        if (owner != DYN_NO_BODY) {
            float4 a = w.aabb[2 * i], b = w.aabb[2 * i + 1];
            f3 mn = xyz(a), mx = xyz(b);
            uint32_t level = shape_levels(mn, mx, base);
            w.c_level[i] = level;
            const BodyHot& h = w.hot[owner];
            bool mv = moves(h.pos.w, h.aux.y);
            bool awake = w.activity[owner] != 0u || w.wake_flags[owner] != 0u;
            run = grid_run(mv, awake);
            float cs = level_size(level, base);
            I3 lo = floor_div(mn, cs), hi = floor_div(mx, cs);
            uint32_t count = (uint32_t)(hi.x - lo.x + 1) * (uint32_t)(hi.y - lo.y + 1) * (uint32_t)(hi.z - lo.z + 1);
            emitted = min(count, DYN_MAX_CELLS_PER_COLLIDER);
            if (count > emitted) add_counter(&w.counters[DYN_COUNTER_ENTRY_FAULTS], count - emitted);
            if (level > 0u && awake) add_counter(&w.counters[DYN_COUNTER_COARSE_ACTIVE], 1u);
            // aggregated updates need one target per coalesced group: branch first
            if (run == RUN_AWAKE) {
                or_counter(&w.counters[DYN_COUNTER_GRID_LEVELS], 1u << level);
                add_counter(&w.counters[DYN_COUNTER_ENTRIES], emitted);
            } else if (run == RUN_RESTING) {
                or_counter(&w.counters[DYN_COUNTER_RESTING_LEVELS], 1u << level);
                add_counter(&w.counters[DYN_COUNTER_RESTING_ENTRIES], emitted);
            } else {
                or_counter(&w.counters[DYN_COUNTER_IMMOVABLE_LEVELS], 1u << level);
                add_counter(&w.counters[DYN_COUNTER_IMMOVABLE_ENTRIES], emitted);
            }
            if (kStep && run != RUN_AWAKE) {
                const float4 first_lo = w.entries[16u * i], first_hi = w.entries[16u * i + 1u];
                const bool kept = w.c_held[i] == run && same_bits(mn, first_lo) && same_bits(mx, first_hi) &&
                                  __float_as_uint(first_lo.w) == owner &&
                                  __float_as_uint(first_hi.w) == entry_info(i, 0u, mv, false);
                if (!kept) stale |= 1u << run;
            }
        }
        if (kStep) {
            const uint32_t held = w.c_held[i];
            if (held != RUN_AWAKE && held != run) stale |= 1u << held;
            w.c_run[i] = run;
            w.run_count[i] = run == RUN_AWAKE ? emitted : 0u;
            w.run_count[w.k + i] = run == RUN_IMMOVABLE ? emitted : 0u;
            w.run_count[2u * w.k + i] = run == RUN_RESTING ? emitted : 0u;
        } else {
            w.entry_count[i] = emitted;
        }
    }
    if (kStep) {
        stale = __reduce_or_sync(0xFFFFFFFFu, stale);
        if ((threadIdx.x & 31u) == 0u && stale != 0u) atomicOr(&w.held[HELD_STALE], stale);
    }
}

// grid_resting_gate.wgsl / grid_resting_commit.wgsl in one thread: which kept runs this step emits
// again (a stale member, or a grid resolution other than the one they were emitted at), the sizes
// and counts the sorts and merge read, and the counters of what was derived. A kept run has exactly
// the entries its members count now, rebuilt or not.
__global__ void k_grid_gate(DeviceWorld w) {
    if (threadIdx.x != 0u) return;
    uint32_t stale = w.held[HELD_STALE];
    w.held[HELD_AWAKE] = w.k ? w.run_offset[w.k - 1u] + w.run_count[w.k - 1u] : 0u;
    const uint32_t base = __float_as_uint(base_cell(w));
    if (base != w.held[HELD_BASE]) stale |= (1u << RUN_IMMOVABLE) | (1u << RUN_RESTING);
    const bool immovable = (stale >> RUN_IMMOVABLE) & 1u, resting = (stale >> RUN_RESTING) & 1u;
    const uint32_t ni = w.counters[DYN_COUNTER_IMMOVABLE_ENTRIES], nr = w.counters[DYN_COUNTER_RESTING_ENTRIES];
    w.held[HELD_STALE] = stale;
    w.held[HELD_BASE] = base;
    w.held[HELD_IMMOVABLE] = ni;
    w.held[HELD_RESTING] = nr;
    w.held[HELD_SORT_IMMOVABLE] = immovable ? ni : 0u;
    w.held[HELD_SORT_RESTING] = resting ? nr : 0u;
    w.counters[DYN_COUNTER_IMMOVABLE_EMITTED] = immovable ? ni : 0u;
    w.counters[DYN_COUNTER_RESTING_REBUILD] = resting ? 1u : 0u;
    w.counters[DYN_COUNTER_RESTING_SORT] = resting ? nr : 0u;
    w.ctl[CTL_ENTRIES] = min(w.held[HELD_AWAKE] + ni + nr, w.e_cap);
    // an empty awake run over kept runs that the last merge already listed alone: the merged list,
    // its cell table and run extents stand as they are (a resting world merges nothing)
    const bool empty = w.held[HELD_AWAKE] == 0u;
    w.held[HELD_LIST_KEPT] = (empty && !immovable && !resting && w.held[HELD_LIST_CLEAN] != 0u) ? 1u : 0u;
    w.held[HELD_LIST_CLEAN] = empty ? 1u : 0u;
}

// collider_emit.wgsl:31-63 for the colliders whose entries this launch writes, in collider order at
// their scanned key positions. A step writes the awake run and every kept run the gate marked
// stale, each entry into its collider's own slots (8 * collider + ordinal), and records which kept
// run a collider's slots now hold. A query writes every collider's entries compactly.
template <bool kStep>
__global__ void k_entry_emit(DeviceWorld w) {
    float base = base_cell(w);
    const uint32_t stale = kStep ? w.held[HELD_STALE] : 0u;
    GRID_STRIDE(i, w.k) {
        uint32_t emitted, first;
        uint32_t* keys;
        uint32_t* vals;
        if (kStep) {
            const uint32_t run = w.c_run[i];
            if (run == RUN_NONE) {
                w.c_held[i] = RUN_AWAKE;
                continue;
            }
            if (run != RUN_AWAKE && ((stale >> run) & 1u) == 0u) continue;  // kept: its slots hold these entries
            w.c_held[i] = run;
            emitted = w.run_count[run * w.k + i];
            first = w.run_offset[run * w.k + i] - (run != RUN_AWAKE ? w.run_offset[run * w.k] : 0u);
            keys = w.run_key + (size_t)run * w.e_cap;
            vals = w.run_val + (size_t)run * w.e_cap;
        } else {
            emitted = w.entry_count[i];
            first = w.entry_offset[i];
            keys = w.ekey;
            vals = w.eval;
        }
        if (emitted == 0u) continue;
        uint32_t owner = w.c_owner[i];
        float4 a = w.aabb[2 * i], b = w.aabb[2 * i + 1];
        f3 mn = xyz(a), mx = xyz(b);
        uint32_t level = w.c_level[i];
        float cs = level_size(level, base);
        I3 lo = floor_div(mn, cs), hi = floor_div(mx, cs);
        uint32_t sy = (uint32_t)(hi.y - lo.y + 1), sz = (uint32_t)(hi.z - lo.z + 1);
        uint32_t rows = sy * sz;
        const BodyHot& h = w.hot[owner];
        bool mv = moves(h.pos.w, h.aux.y);
        bool awake = w.activity[owner] != 0u || w.wake_flags[owner] != 0u;
        const uint32_t world = w.body_world[owner];
        for (uint32_t ordinal = 0; ordinal < emitted; ++ordinal) {
            I3 c = I3{lo.x + (int)(ordinal / rows), lo.y + (int)((ordinal / sz) % sy), lo.z + (int)(ordinal % sz)};
            uint32_t offset = (uint32_t)(c.x - lo.x) | ((uint32_t)(c.y - lo.y) << 1) | ((uint32_t)(c.z - lo.z) << 2);
            uint32_t slot = kStep ? 8u * i + ordinal : first + ordinal;
            keys[first + ordinal] = cell_key_in(level, c, world);
            vals[first + ordinal] = slot;
            w.entries[2 * slot] = make_float4(mn.x, mn.y, mn.z, __uint_as_float(owner));
            w.entries[2 * slot + 1] = make_float4(mx.x, mx.y, mx.z, __uint_as_float(entry_info(i, offset, mv, awake)));
        }
    }
}

// Entries of a run sorted by (cell key, slot) that come before (key, slot).
__device__ __forceinline__ uint32_t run_rank(const uint32_t* keys, const uint32_t* vals, uint32_t n, uint32_t key,
                                             uint32_t val) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t k = __ldg(keys + mid);
        if (k < key || (k == key && __ldg(vals + mid) < val)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// The three sorted runs merged into the entry list the cell table and the pair kernels read. Each
// run is sorted by cell key and, within a key, by slot (its keys were scanned in collider and cell
// order and the sort is stable), so an entry's place is its index in its run plus the entries of
// the other runs before (key, slot): the list one sort of every entry would give.
__global__ void k_entry_merge(DeviceWorld w) {
    if (w.held[HELD_LIST_KEPT] != 0u) return;
    const uint32_t na = w.held[HELD_AWAKE], ni = w.held[HELD_IMMOVABLE], nr = w.held[HELD_RESTING];
    const uint32_t total = min(na + ni + nr, w.e_cap);
    const uint32_t* ka = w.run_key;
    const uint32_t* va = w.run_val;
    const uint32_t* ki = w.run_key + w.e_cap;
    const uint32_t* vi = w.run_val + w.e_cap;
    const uint32_t* kr = w.run_key + 2u * (size_t)w.e_cap;
    const uint32_t* vr = w.run_val + 2u * (size_t)w.e_cap;
    GRID_STRIDE(t, total) {
        uint32_t key, val, pos;
        if (t < na) {
            key = __ldg(ka + t);
            val = __ldg(va + t);
            pos = t + run_rank(ki, vi, ni, key, val) + run_rank(kr, vr, nr, key, val);
        } else if (t < na + ni) {
            const uint32_t j = t - na;
            key = __ldg(ki + j);
            val = __ldg(vi + j);
            pos = j + run_rank(ka, va, na, key, val) + run_rank(kr, vr, nr, key, val);
        } else {
            const uint32_t j = t - na - ni;
            key = __ldg(kr + j);
            val = __ldg(vr + j);
            pos = j + run_rank(ka, va, na, key, val) + run_rank(ki, vi, ni, key, val);
        }
        if (pos < w.e_cap) {
            w.ekey[pos] = key;
            w.eval[pos] = val;
        }
        if (t < na + ni) w.init_pos[t] = pos;
    }
}

// ---- pair emission (cell_pairs.wgsl, level_links.wgsl, pair_emit.wgsl) ----
struct GEntry {
    f3 mn, mx;
    uint32_t group, info;
};
__device__ __forceinline__ GEntry load_entry(const DeviceWorld& w, uint32_t node) {
    float4 a = w.entries[2 * node], b = w.entries[2 * node + 1];
    return GEntry{xyz(a), xyz(b), __float_as_uint(a.w), __float_as_uint(b.w)};
}
__device__ __forceinline__ bool entry_awake(const DeviceWorld& w, const GEntry& e) {
    if ((e.info & DYN_ENTRY_MOBILE) == 0u) return w.wake_flags[e.group] != 0u;
    return (e.info & DYN_ENTRY_AWAKE) != 0u;
}
__device__ __forceinline__ bool overlaps(const GEntry& a, const GEntry& b) {
    return a.mn.x <= b.mx.x && a.mn.y <= b.mx.y && a.mn.z <= b.mx.z && b.mn.x <= a.mx.x && b.mn.y <= a.mx.y && b.mn.z <= a.mx.z;
}
__device__ __forceinline__ I3 entry_cell(const GEntry& e, float cs) {
    uint32_t bits = (e.info & DYN_ENTRY_CELL_MASK) >> DYN_ENTRY_CELL_SHIFT;
    I3 c = floor_div(e.mn, cs);
    return I3{c.x + (int)(bits & 1u), c.y + (int)((bits >> 1) & 1u), c.z + (int)((bits >> 2) & 1u)};
}
__device__ __forceinline__ bool same_cell(I3 a, I3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
__device__ __forceinline__ bool overlap_cell_is(const GEntry& a, const GEntry& b, float cs, I3 cell) {
    return same_cell(floor_div(vmax(a.mn, b.mn), cs), cell);
}
__device__ __forceinline__ void emit_pair(const DeviceWorld& w, const GEntry& a, const GEntry& b, bool same_node) {
    if (((a.info & DYN_ENTRY_KIND_MASK) >> DYN_ENTRY_KIND_SHIFT) != DYN_ENTRY_KIND_COLLIDER) return;
    if (((b.info & DYN_ENTRY_KIND_MASK) >> DYN_ENTRY_KIND_SHIFT) != DYN_ENTRY_KIND_COLLIDER) return;
    if (same_node || a.group == b.group) return;
    if ((a.info & DYN_ENTRY_MOBILE) == 0u && (b.info & DYN_ENTRY_MOBILE) == 0u) return;
    if (w.body_world[a.group] != w.body_world[b.group]) return;  // different sub-worlds of a batch
    uint32_t slot = append_slot(&w.counters[DYN_COUNTER_PAIRS]);
    if (slot < w.p_cap) {
        uint32_t ia = a.info & DYN_ENTRY_INDEX_MASK, ib = b.info & DYN_ENTRY_INDEX_MASK;
        w.pmaj[slot] = min(ia, ib);
        w.pmin[slot] = max(ia, ib);
    } else {
        add_counter(&w.counters[DYN_COUNTER_REFUSED_PAIRS], 1u);
    }
}
__device__ __forceinline__ uint32_t lower_bound(const uint32_t* keys, uint32_t n, uint32_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(keys + mid) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// ---- cell table: cell key -> first index of its run in the sorted entries ----
// An open-addressing table rebuilt every step after the entry sort, sized to twice the live entry
// count (a power of two, at most 1 << cell_bits), so the coarse-level walk of k_pairs finds a cell
// in one or two probes instead of a binary search over all entries. Key 0xFFFFFFFF marks an empty
// slot; no cell key reaches it (levels stop at DYN_GRID_LEVEL_LIMIT). If an insert ever fails its
// bounded probe, CTL_CELL_OVERFLOW is set and every lookup of that step searches the sorted keys
// instead, so the pairs found never depend on the table.
constexpr uint32_t kCellEmpty = 0xFFFFFFFFu;
constexpr uint32_t kCellProbeLimit = 1024u;
__device__ __forceinline__ uint32_t cell_table_bits(const DeviceWorld& w, uint32_t live) {
    uint32_t bits = 10u;
    while (bits < w.cell_bits && (1u << bits) < 2u * live) ++bits;
    return bits;
}
__device__ __forceinline__ uint32_t cell_slot(uint32_t key, uint32_t bits) { return (key * 0x9E3779B1u) >> (32u - bits); }

__global__ void k_cell_clear(DeviceWorld w) {
    if (w.held[HELD_LIST_KEPT] != 0u) return;
    const uint32_t live = min(w.ctl[CTL_ENTRIES], w.e_cap);
    const uint32_t slots = 1u << cell_table_bits(w, live);
    GRID_STRIDE(i, slots) w.cell_table[i] = make_uint2(kCellEmpty, 0u);
}

__global__ void k_cell_insert(DeviceWorld w) {
    if (w.held[HELD_LIST_KEPT] != 0u) return;
    const uint32_t live = min(w.ctl[CTL_ENTRIES], w.e_cap);
    const uint32_t bits = cell_table_bits(w, live);
    const uint32_t mask = (1u << bits) - 1u;
    GRID_STRIDE(i, live) {
        uint32_t key = w.ekey[i];
        if (i > 0u && w.ekey[i - 1u] == key) continue;
        // the run's extent for every member, so the pair kernels walk a run without testing keys
        uint32_t end = i + 1u;
        while (end < live && w.ekey[end] == key) ++end;
        for (uint32_t t = i; t < end; ++t) w.erun[t] = make_uint2(i, end - i);
        uint32_t slot = cell_slot(key, bits);
        bool placed = false;
        for (uint32_t probe = 0; probe < kCellProbeLimit; ++probe) {
            if (atomicCAS(&w.cell_table[slot].x, kCellEmpty, key) == kCellEmpty) {
                w.cell_table[slot].y = i;
                placed = true;
                break;
            }
            slot = (slot + 1u) & mask;
        }
        if (!placed) atomicOr(&w.ctl[CTL_CELL_OVERFLOW], 1u);
    }
}

// First index of the run of `key` in the sorted entries, or `live` when no entry has it.
__device__ __forceinline__ uint32_t cell_find(const DeviceWorld& w, uint32_t live, uint32_t bits, bool overflow, uint32_t key) {
    if (overflow) {
        uint32_t j = lower_bound(w.ekey, live, key);
        return (j < live && __ldg(w.ekey + j) == key) ? j : live;
    }
    const uint32_t mask = (1u << bits) - 1u;
    uint32_t slot = cell_slot(key, bits);
    for (uint32_t probe = 0; probe < kCellProbeLimit; ++probe) {
        uint2 e = __ldg(w.cell_table + slot);
        if (e.x == key) return e.y;
        if (e.x == kCellEmpty) return live;
        slot = (slot + 1u) & mask;
    }
    return live;
}

// Pair emission in two kernels whose warps each do one kind of work: the coarse-level links of
// every collider's primary entry (level_links.wgsl:6-65; one thread per collider, whose primary entry
// is its first emitted slot), and the same-cell mates of every sorted entry (cell_pairs.wgsl:6-50).
// The pair set does not depend on which kernel emits a pair first: the list is sorted afterwards.
//
// The coarse links spread over gridDim.y: thread (i, y) walks collider i's cells at the occupied
// levels whose rank among the occupied levels is y, y + gridDim.y, ... (the walk of one collider is
// a chain of dependent lookups; splitting it by level shortens the chain a thread waits through).
constexpr uint32_t kCoarseLevelSlices = 4u;
constexpr uint32_t kRunBatch = 4u;            // entries of a cell run the coarse walk loads together
constexpr uint32_t kCellBatch = 2u;           // the same for the same-cell scan, whose runs are short
constexpr uint32_t kNoEntry = 0xFFFFFFFFu;
__global__ void __launch_bounds__(128) k_pairs_coarse(DeviceWorld w) {
    const uint32_t live = min(w.ctl[CTL_ENTRIES], w.e_cap);
    const float grid = base_cell(w);
    const uint32_t occupied =
        w.counters[DYN_COUNTER_GRID_LEVELS] | w.counters[DYN_COUNTER_RESTING_LEVELS] | w.counters[DYN_COUNTER_IMMOVABLE_LEVELS];
    const bool coarse_active = w.counters[DYN_COUNTER_COARSE_ACTIVE] != 0u;
    const uint32_t bits = cell_table_bits(w, live);
    const bool overflow = w.ctl[CTL_CELL_OVERFLOW] != 0u;
    GRID_STRIDE(i, w.k) {
        if (w.c_run[i] == RUN_NONE) continue;
        const uint32_t node = 8u * i;  // the first of the collider's slots: its primary entry
        GEntry e = load_entry(w, node);
        if (((e.info & DYN_ENTRY_KIND_MASK) >> DYN_ENTRY_KIND_SHIFT) != DYN_ENTRY_KIND_COLLIDER) continue;
        if ((e.info & DYN_ENTRY_PRIMARY) == 0u) continue;
        const bool awake = entry_awake(w, e);
        if (!(awake || coarse_active)) continue;
        const uint32_t level = w.c_level[e.info & DYN_ENTRY_INDEX_MASK];
        const uint32_t world = w.body_world[e.group];
        const uint32_t coarser = occupied & ~((1u << min(level + 1u, 31u)) - 1u);
        // the levels of this slice: every gridDim.y-th set bit of `coarser`, from the lowest
        uint32_t rest = coarser;
        for (uint32_t skip = 0; skip < blockIdx.y && rest != 0u; ++skip) rest &= rest - 1u;
        while (rest != 0u) {
            const uint32_t link = (uint32_t)__ffs(rest) - 1u;
            for (uint32_t skip = 0; skip < gridDim.y && rest != 0u; ++skip) rest &= rest - 1u;
            float cs = level_size(link, grid);
            I3 lo = floor_div(e.mn, cs), hi = floor_div(e.mx, cs);
            // A box spans at most two cells per axis at any level coarser than its own; a wider
            // span only comes from a non-finite box, whose walk is cut short and counted.
            if ((long long)hi.x - lo.x > 3 || (long long)hi.y - lo.y > 3 || (long long)hi.z - lo.z > 3 || hi.x < lo.x ||
                hi.y < lo.y || hi.z < lo.z) {
                add_counter(&w.counters[DYN_COUNTER_ENTRY_FAULTS], 1u);
                continue;
            }
            for (int x = lo.x; x <= hi.x; ++x)
                for (int y = lo.y; y <= hi.y; ++y)
                    for (int z = lo.z; z <= hi.z; ++z) {
                        I3 cell = I3{x, y, z};
                        uint32_t key = cell_key_in(link, cell, world);
                        uint32_t j = cell_find(w, live, bits, overflow, key);
                        if (j >= live) continue;
                        const uint32_t end = j + __ldg(&w.erun[j].y);
                        // the run's entries four at a time: their loads are independent, so they
                        // are all in flight before the first test
                        for (; j < end; j += kRunBatch) {
                            uint32_t others[kRunBatch];
                            GEntry o[kRunBatch];
#pragma unroll
                            for (uint32_t u = 0; u < kRunBatch; ++u) others[u] = j + u < end ? __ldg(w.eval + j + u) : node;
#pragma unroll
                            for (uint32_t u = 0; u < kRunBatch; ++u) {
                                if (others[u] != node) o[u] = load_entry(w, others[u]);
                            }
#pragma unroll
                            for (uint32_t u = 0; u < kRunBatch; ++u) {
                                if (others[u] == node) continue;
                                if (!awake && !entry_awake(w, o[u])) continue;
                                if (!overlaps(e, o[u])) continue;
                                if (!same_cell(entry_cell(o[u], cs), cell)) continue;
                                if (!overlap_cell_is(e, o[u], cs, cell)) continue;
                                emit_pair(w, e, o[u], false);
                            }
                        }
                    }
        }
    }
}

// One thread per entry that can start a pair (an awake entry, or an immovable one, whose owner's
// wake flag makes it awake): a resting entry is never awake, so it only answers.
__global__ void k_pairs_cell(DeviceWorld w) {
    const uint32_t live = min(w.ctl[CTL_ENTRIES], w.e_cap);
    const uint32_t starts = min(w.held[HELD_AWAKE] + w.held[HELD_IMMOVABLE], live);
    const float grid = base_cell(w);
    GRID_STRIDE(t, starts) {
        const uint32_t index = __ldg(w.init_pos + t);
        uint32_t node = w.eval[index];
        GEntry e = load_entry(w, node);
        if (((e.info & DYN_ENTRY_KIND_MASK) >> DYN_ENTRY_KIND_SHIFT) != DYN_ENTRY_KIND_COLLIDER) continue;
        if (!entry_awake(w, e)) continue;
        uint32_t level = w.c_level[e.info & DYN_ENTRY_INDEX_MASK];
        float cs = level_size(level, grid);
        I3 cell = entry_cell(e, cs);
        const uint2 run = __ldg(&w.erun[index]);
        const uint32_t end = run.x + run.y;
        for (uint32_t j = run.x; j < end; j += kCellBatch) {
            uint32_t others[kCellBatch];
            GEntry o[kCellBatch];
#pragma unroll
            for (uint32_t u = 0; u < kCellBatch; ++u) others[u] = (j + u < end && j + u != index) ? __ldg(w.eval + j + u) : kNoEntry;
#pragma unroll
            for (uint32_t u = 0; u < kCellBatch; ++u) {
                if (others[u] != kNoEntry) o[u] = load_entry(w, others[u]);
            }
#pragma unroll
            for (uint32_t u = 0; u < kCellBatch; ++u) {
                if (others[u] == kNoEntry) continue;
                if (j + u < index && entry_awake(w, o[u])) continue;
                if (!overlaps(e, o[u])) continue;
                if (!same_cell(entry_cell(o[u], cs), cell)) continue;
                if (!overlap_cell_is(e, o[u], cs, cell)) continue;
                emit_pair(w, e, o[u], node == others[u]);
            }
        }
    }
}

// ---- narrowphase (narrowphase.wgsl:518-685) into the staging set, then ordered compaction ----
__device__ __forceinline__ void write_contact(const ContactSet& s, uint32_t cap, uint32_t i, const Mani& m, uint32_t ra,
                                              uint32_t rb, uint32_t ca, uint32_t cb, const DBody& fb, const DBody& sb,
                                              uint32_t fid, uint32_t sid, uint32_t fgen, uint32_t sgen, bool sensor,
                                              float4 fmat, float4 smat, float4 fmat2, float4 smat2, uint32_t fflags,
                                              uint32_t sflags, uint32_t fcomb, uint32_t rcomb) {
    auto combine = [](float a, float b, uint32_t mode) -> float {
        if (mode == 1u) return wmin(a, b);
        if (mode == 2u) return wmax(a, b);
        if (mode == 3u) return (a + b) * 0.5f;
        return sqrtf(a * b);
    };
    float friction = combine(fmat.x, smat.x, fcomb);
    float restitution = combine(fmat.y, smat.y, rcomb);
    uint32_t events = (fflags & sflags) & (DYN_EVENT_MODE_BEGIN_END | DYN_EVENT_MODE_PERSIST);
    s.normal[i] = mk4(m.normal, friction);
    s.rows[i] = make_uint4(ra, rb, m.count | ((sensor ? 1u : 0u) << 8), events);
    s.mat[i] = make_float4(wmax(fmat.z, smat.z), wmax(fmat.w, smat.w), fmat2.x + smat2.x, wmax(fmat2.y, smat2.y));
    s.ids[i] = make_uint4(ca, cb, fid, sid);
    s.ids2[i] = make_uint4(fgen, sgen, DYN_NO_SURFACE, DYN_NO_TRIANGLE);
    s.extra[i] = make_float4(restitution, 0.0f, 0.0f, 0.0f);
    for (uint32_t p = 0; p < m.count; ++p) {
        f3 point = m.p[p].position;
        f3 la = quat_rotate(quat_conj(fb.orientation), point - fb.position);
        f3 lb = quat_rotate(quat_conj(sb.orientation), point - sb.position);
        size_t o = (size_t)p * cap + i;
        s.la[o] = mk4(la, m.p[p].depth);
        s.lb[o] = mk4(lb, 0.0f);
        s.acc[o] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(m.p[p].feature));
        s.pos[o] = mk4(point, 0.0f);
    }
}

enum PairClass : uint32_t { PC_ANALYTIC = 0, PC_BOXES = 1, PC_CONVEX = 2, PC_COUNT = 3 };

// narrowphase.wgsl:518-550 (filters) then the shape dispatch of :551-652, decided once per pair:
// pairs that fail a filter are answered here; the rest go to one list per kernel class.
// joined_pairs.wgsl: is there an unbroken joint between these rows that disables their collisions?
// jfilter is sorted by (lower row, higher row); several joints may join one pair.
__device__ __forceinline__ bool joined_by_joint(const DeviceWorld& w, uint32_t ra, uint32_t rb) {
    const uint32_t count = w.jfilter_count;
    if (count == 0u) return false;
    const uint32_t a = min(ra, rb), b = max(ra, rb);
    uint32_t lo = 0, hi = count;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint2 e = w.jfilter[mid];
        if (e.x < a || (e.x == a && e.y < b)) {
            lo = mid + 1u;
        } else {
            hi = mid;
        }
    }
    for (; lo < count; ++lo) {
        const uint2 e = w.jfilter[lo];
        if (e.x != a || e.y != b) break;
        if (w.jruntime[w.jfilter_joint[lo]].broken == 0u) return true;
    }
    return false;
}

__global__ void k_pair_class(DeviceWorld w) {
    const uint32_t pairs = min(w.counters[DYN_COUNTER_PAIRS], w.p_cap);
    GRID_STRIDE(index, pairs) {
        const uint4 f = w.c_class[w.pmaj[index]], s = w.c_class[w.pmin[index]];
        const uint32_t fr = f.x, sr = s.x, fk = f.w & 0xffu, sk = s.w & 0xffu;
        int cls = -1;
        do {
            if (fr == DYN_NO_BODY || sr == DYN_NO_BODY || fr == sr) break;
            if (((f.w | s.w) & 0x100u) == 0u) break;  // neither body moves
            if (fk == 0u || sk == 0u) break;
            if (!((f.y & s.z) != 0u && (s.y & f.z) != 0u)) break;
            if (joined_by_joint(w, fr, sr)) break;
            bool fw = shape_world_geometry(fk), sw = shape_world_geometry(sk);
            if (fw && sw) break;
            if (fw || sw) {
                if ((fw ? fk : sk) != 9u) break;  // meshes and heightfields are outside this path
                cls = PC_ANALYTIC;                // plane against a convex: one feature ring
                break;
            }
            bool unscaled = (f.w & s.w & 0x200u) != 0u;
            if (!unscaled || !shape_analytic(fk) || !shape_analytic(sk) || (fk == 2u && sk == 3u) || (fk == 3u && sk == 2u)) {
                cls = PC_CONVEX;
            } else if (fk == 2u && sk == 2u) {
                cls = PC_BOXES;
            } else {
                cls = PC_ANALYTIC;
            }
        } while (false);
        if (cls < 0) {
            continue;  // answered here: no contact
        } else if (cls == PC_ANALYTIC) {  // one branch per list: an aggregated append needs one target
            w.np_list[append_slot(&w.ctl[CTL_LIST0 + PC_ANALYTIC])] = index;
        } else if (cls == PC_BOXES) {
            w.np_list[(size_t)PC_BOXES * w.p_cap + append_slot(&w.ctl[CTL_LIST0 + PC_BOXES])] = index;
        } else {
            w.np_list[(size_t)PC_CONVEX * w.p_cap + append_slot(&w.ctl[CTL_LIST0 + PC_CONVEX])] = index;
        }
    }
}

// One pair of a class list through its narrowphase kernel (the pair passed the filters).
template <int kClass>
__device__ __forceinline__ void narrow_pair(const DeviceWorld& w, const dyn_step_params& p, uint32_t index) {
    uint32_t fs = w.pmaj[index], ss = w.pmin[index];
    uint32_t fr = w.c_owner[fs], sr = w.c_owner[ss];
    DBody fb = load_dbody(w.hot, fr), sb = load_dbody(w.hot, sr);
    DColl fc = load_dcoll(w, fs), sc = load_dcoll(w, ss);
    uint4 fi = w.ident[fr], si = w.ident[sr];
    bool sensor = (fc.flags & DYN_COLLIDER_SENSOR) != 0u || (sc.flags & DYN_COLLIDER_SENSOR) != 0u;
    float margin = p.contact_margin;
    if ((fb.flags & DYN_BODY_CCD) || (sb.flags & DYN_BODY_CCD)) {
        margin = p.contact_margin + length(sb.velocity - fb.velocity) * p.dt;
    }
    Mani m;
    m.count = 0;
    m.normal = s3(0.0f);
    if (kClass == PC_ANALYTIC) {
        if (fc.kind == 9u) {
            m = plane_convex(w, world_shape(fb.position, fb.orientation, fc), world_shape(sb.position, sb.orientation, sc), margin);
        } else if (sc.kind == 9u) {
            m = plane_convex(w, world_shape(sb.position, sb.orientation, sc), world_shape(fb.position, fb.orientation, fc), margin);
            m.normal = -m.normal;
            for (uint32_t q = 0; q < m.count; ++q) m.p[q].feature = feature_mirror(m.p[q].feature);
        } else if (fc.kind == 1u && sc.kind == 1u) {
            m = sphere_sphere(fb, fc, sb, sc, margin);
        } else if (fc.kind == 1u && sc.kind == 2u) {
            m = sphere_box(fb, fc, sb, sc, margin);
        } else if (fc.kind == 1u && sc.kind == 3u) {
            m = sphere_capsule(fb, fc, sb, sc, margin);
        } else if (fc.kind == 2u && sc.kind == 1u) {
            m = sphere_box(sb, sc, fb, fc, margin);
            m.normal = -m.normal;
        } else if (fc.kind == 3u && sc.kind == 1u) {
            m = sphere_capsule(sb, sc, fb, fc, margin);
            m.normal = -m.normal;
        } else {
            m = capsule_capsule(fb, fc, sb, sc, margin);
        }
    } else if (kClass == PC_BOXES) {
        m = box_box_sat(fb, fc, sb, sc, margin);
    } else {
        WShape a = world_shape(fb.position, fb.orientation, fc);
        WShape b = world_shape(sb.position, sb.orientation, sc);
        Hit hit = convex_hit(w, a, b);
        if (hit.distance <= margin) {
            mani_emit(&m, hit.normal);
            if (!convex_pair_manifold(w, a, b, hit.normal, &m)) mani_push(&m, hit.point, -hit.distance, kFeatPoint);
        }
    }
    if (m.count > 0u) {
        uint32_t slot = append_slot(&w.ctl[CTL_APPENDED]);
        if (slot < w.s_cap) {
            write_contact(w.tmp, w.s_cap, slot, m, fr, sr, fs, ss, fb, sb, fi.x, si.x, fi.y, si.y, sensor, w.c_mat[fs],
                          w.c_mat[ss], w.c_mat2[fs], w.c_mat2[ss], fc.flags, sc.flags, p.friction_combine,
                          p.restitution_combine);
        } else {
            add_counter(&w.counters[DYN_COUNTER_REFUSED_CONTACTS], 1u);
        }
    }
}

// ---- the convex class in three phases ----
__device__ __forceinline__ float pair_margin(const dyn_step_params& p, const DBody& fb, const DBody& sb) {
    if ((fb.flags & DYN_BODY_CCD) || (sb.flags & DYN_BODY_CCD)) return p.contact_margin + length(sb.velocity - fb.velocity) * p.dt;
    return p.contact_margin;
}
__device__ __forceinline__ void convex_shapes(const DeviceWorld& w, uint32_t index, WShape* a, WShape* b, DBody* fb, DBody* sb) {
    uint32_t fs = w.pmaj[index], ss = w.pmin[index];
    *fb = load_dbody(w.hot, w.c_owner[fs]);
    *sb = load_dbody(w.hot, w.c_owner[ss]);
    DColl fc = load_dcoll(w, fs), sc = load_dcoll(w, ss);
    *a = world_shape(fb->position, fb->orientation, fc);
    *b = world_shape(sb->position, sb->orientation, sc);
}
__device__ __forceinline__ void push_hit(const DeviceWorld& w, uint32_t index, const Hit& hit) {
    uint32_t slot = append_slot(&w.ctl[CTL_HITS]);
    w.hit_list[slot] = index;
    w.hit_data[2 * (size_t)slot] = mk4(hit.point, hit.distance);
    w.hit_data[2 * (size_t)slot + 1] = mk4(hit.normal, 0.0f);
}

// Slack above the contact margin before a pair is rejected on its centre-axis gap alone: well above
// the rounding of support points at world coordinates of a few hundred metres (~1e-5 m).
constexpr float kRejectTolerance = 1e-3f;

// Phase 1: GJK per pair (convex.wgsl:464-521) and, for separated shapes, the penetration probe
// (convex.wgsl:532-582, 588-600); penetrating pairs queue for EPA.
//
// The work of one pair is a sequence of support-pair evaluations: the first along the centre axis,
// one per GJK iteration along -v, up to three that grow a penetrating simplex to a tetrahedron, and
// one per probe direction. Each lane runs its pair as a state machine that makes exactly one
// support-pair evaluation per trip of the loop below, and a lane whose pair is done takes the next
// pair from the convex list through a shared ticket. So the lanes of a warp keep evaluating
// supports together instead of waiting for the warp's slowest pair, whatever their pairs' iteration
// counts. Each state does the same arithmetic, in the same order, as gjk_phase followed by
// separated_hit (narrow.cuh); only the interleaving of pairs on a lane changes.
enum GjkState : uint32_t { GS_IDLE = 0, GS_FIRST = 1, GS_ITER = 2, GS_EXPAND = 3 };
// simplex triples in the probe's order (i < j < k ascending), one per bit of GjkLane::triples
__constant__ uint8_t kProbeTriple[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
constexpr uint32_t kProbeCentre = 4u, kProbeAxes = 5u, kProbeEnd = 11u;

struct GjkLane {
    uint32_t state, index, count, iter;
    float tiny, margin, dist;
    f3 pa, pb, normal;
    SPt* s;  // the simplex (4 points), in this lane's slice of shared memory
    SRes cl;
    WShape a, b;
};
// Each lane's simplex lives in shared memory at an odd word stride (37 words for 36 used), so the
// lanes of a warp reading the same point land in different banks; held in the lane's registers it
// would be indexed by the simplex size and spill to local memory.
constexpr uint32_t kGjkThreads = 128;
constexpr uint32_t kSimplexStride = 37;
static_assert(sizeof(SPt) * 4 <= kSimplexStride * sizeof(float), "a lane's simplex fits its slice");

// A pair that GJK leaves separated, or that runs out of iterations, goes to the penetration probe's
// queue with its simplex, its closest points and its normal (k_convex_probe).
__device__ __forceinline__ void gjk_to_probe(const DeviceWorld& w, GjkLane& L) {
    const uint32_t slot = append_slot(&w.ctl[CTL_PROBES]);
    w.probe_list[slot] = L.index;
    float4* q = w.probe_data + 6 * (size_t)slot;
    q[0] = mk4(L.s[0].w, __uint_as_float(L.count));
    q[1] = mk4(L.count > 1u ? L.s[1].w : s3(0.0f), L.dist);
    q[2] = mk4(L.count > 2u ? L.s[2].w : s3(0.0f), L.pa.x);
    q[3] = mk4(L.count > 3u ? L.s[3].w : s3(0.0f), L.pa.y);
    q[4] = mk4(L.pb, L.pa.z);
    q[5] = mk4(L.normal, 0.0f);
    L.state = GS_IDLE;
}
// A penetrating pair with its tetrahedron complete goes to the EPA queue.
__device__ __forceinline__ void gjk_to_epa(const DeviceWorld& w, GjkLane& L) {
    const uint32_t slot = append_slot(&w.ctl[CTL_EPA]);
    w.epa_list[slot] = L.index;
    for (uint32_t k = 0; k < 4; ++k) w.epa_simplex[4 * (size_t)slot + k] = mk4(L.s[k].w, 0.0f);
    L.state = GS_IDLE;
}
// The loop head of gjk_phase: terminate, grow a penetrating simplex, or take another iteration.
__device__ __forceinline__ void gjk_head(const DeviceWorld& w, GjkLane& L) {
    if (L.iter >= 24u) {
        gjk_to_probe(w, L);
    } else if (L.cl.pen || length(L.cl.v) < L.tiny) {
        if (L.count < 4u) {
            L.state = GS_EXPAND;
        } else {
            gjk_to_epa(w, L);
        }
    } else {
        L.state = GS_ITER;
    }
}
__device__ __forceinline__ void gjk_separated(const DeviceWorld& w, GjkLane& L) {
    L.dist = length(L.cl.v);
    L.pa = L.cl.pa;
    L.pb = L.cl.pb;
    if (L.dist > 1e-6f) L.normal = sign_normalize(L.cl.pb - L.cl.pa);
    gjk_to_probe(w, L);
}

// The centre-axis rejection of gjk_phase for every convex pair, ahead of the state machine: one
// support-pair evaluation per pair with the arithmetic of the state machine's first trip, one thread
// per pair. In a pile about nine convex pairs in ten stop here; the rest go on to k_convex_gjk,
// whose first trip repeats the same test and passes.
__global__ void __launch_bounds__(128) k_convex_reject(DeviceWorld w, dyn_step_params p) {
    const uint32_t count = min(w.ctl[CTL_LIST0 + PC_CONVEX], w.p_cap);
    const uint32_t* list = w.np_list + (size_t)PC_CONVEX * w.p_cap;
    uint32_t* gjk_pairs = w.np_list + (size_t)PC_COUNT * w.p_cap;
    GRID_STRIDE(i, count) {
        const uint32_t index = list[i];
        WShape a, b;
        DBody fb, sb;
        convex_shapes(w, index, &a, &b, &fb, &sb);
        const float margin = pair_margin(p, fb, sb);
        f3 d = b.center - a.center;
        if (length(d) < 1e-8f) d = mk3(1.0f, 0.0f, 0.0f);
        const SPt sp = support_pair(w, a, b, d);
        if (dot(sp.w, d) < -(margin + kRejectTolerance) * length(d)) continue;
        gjk_pairs[append_slot(&w.ctl[CTL_GJK_PAIRS])] = index;
    }
}

__global__ void __launch_bounds__(kGjkThreads, 6) k_convex_gjk(DeviceWorld w, dyn_step_params p) {
    __shared__ float simplex_slices[kGjkThreads * kSimplexStride];
    const uint32_t count = min(w.ctl[CTL_GJK_PAIRS], w.p_cap);
    const uint32_t* list = w.np_list + (size_t)PC_COUNT * w.p_cap;
    GjkLane L;
    L.s = reinterpret_cast<SPt*>(simplex_slices + threadIdx.x * kSimplexStride);
    L.state = GS_IDLE;
    for (;;) {
        if (L.state == GS_IDLE) {
            const uint32_t ticket = append_slot(&w.ctl[CTL_GJK_NEXT]);
            if (ticket >= count) break;
            L.index = list[ticket];
            DBody fb, sb;
            convex_shapes(w, L.index, &L.a, &L.b, &fb, &sb);
            L.margin = pair_margin(p, fb, sb);
            L.count = 0u;
            L.dist = 0.0f;
            L.pa = L.a.center;
            L.pb = L.b.center;
            L.normal = sign_normalize(L.b.center - L.a.center);
            L.state = GS_FIRST;
        }
        f3 d;
        if (L.state == GS_FIRST) {
            d = L.b.center - L.a.center;
            if (length(d) < 1e-8f) d = mk3(1.0f, 0.0f, 0.0f);
        } else if (L.state == GS_ITER) {
            d = -L.cl.v;
        } else {
            d = simplex_expand_dir(L.s, L.count);
        }
        const SPt sp = support_pair(w, L.a, L.b, d);
        if (L.state == GS_FIRST) {
            L.s[0] = sp;
            L.count = 1u;
            // the exact centre-axis rejection of gjk_phase
            if (dot(sp.w, d) < -(L.margin + kRejectTolerance) * length(d)) {
                L.state = GS_IDLE;
                continue;
            }
            L.cl = simplex_closest(L.s, L.count);
            L.tiny = 1e-4f * wmin(shape_scale(L.a), shape_scale(L.b));
            L.iter = 0u;
            gjk_head(w, L);
        } else if (L.state == GS_ITER) {
            const f3 v = L.cl.v;
            if (dot(sp.w, -v) <= dot(v, -v) + 1e-4f * wmax(1.0f, dot(v, v))) {
                gjk_separated(w, L);
                continue;
            }
            // simplex_reduce: keep the points with weight, in order (a stable in-place compaction)
            uint32_t kc = 0;
            for (uint32_t i = 0; i < 4; ++i) {
                if (L.cl.lam[i] > 1e-6f) {
                    if (kc != i) L.s[kc] = L.s[i];
                    ++kc;
                }
            }
            if (kc == 0u) kc = 1;  // no weight: keep the first point
            L.count = kc;
            const float span = shape_scale(L.b);
            const float tol = (1e-5f * span) * (1e-5f * span);
            bool holds = false;
            for (uint32_t i = 0; i < L.count; ++i) {
                const f3 off = L.s[i].w - sp.w;
                if (dot(off, off) <= tol) holds = true;
            }
            if (holds) {
                gjk_separated(w, L);
                continue;
            }
            L.s[L.count] = sp;
            L.count += 1u;
            L.cl = simplex_closest(L.s, L.count);
            L.iter += 1u;
            gjk_head(w, L);
        } else {
            L.s[L.count] = sp;
            L.count += 1u;
            if (L.count == 4u) gjk_to_epa(w, L);
        }
    }
}

// convex.wgsl:532-582 (penetration_probe) then separated_hit (:588-600) for the pairs GJK left
// separated: the simplex triples, the centre axis and the six axes in order, stopping at the first
// direction with no overlap (the minimum is then not positive, which is all separated_hit asks);
// when every direction overlaps, the first minimum gives the penetration. One thread per pair.
__global__ void __launch_bounds__(128) k_convex_probe(DeviceWorld w, dyn_step_params p) {
    const uint32_t count = min(w.ctl[CTL_PROBES], w.p_cap);
    GRID_STRIDE(i, count) {
        const uint32_t index = w.probe_list[i];
        const float4* q = w.probe_data + 6 * (size_t)i;
        const float4 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4], q5 = q[5];
        const f3 sw[4] = {xyz(q0), xyz(q1), xyz(q2), xyz(q3)};
        const uint32_t n = __float_as_uint(q0.w);
        const float dist = q1.w;
        const f3 pa = mk3(q2.w, q3.w, q4.w), pb = xyz(q4), normal = xyz(q5);
        WShape a, b;
        DBody fb, sb;
        convex_shapes(w, index, &a, &b, &fb, &sb);
        const float margin = pair_margin(p, fb, sb);
        uint32_t triples = 0u;
        const uint32_t ntri = n == 3u ? 1u : (n == 4u ? 4u : 0u);
        for (uint32_t t = 0; t < ntri; ++t) {
            const f3 wi = sw[kProbeTriple[t][0]], wj = sw[kProbeTriple[t][1]], wk = sw[kProbeTriple[t][2]];
            if (length(cross(wj - wi, wk - wi)) > 1e-8f) triples |= 1u << t;
        }
        const bool centre = !(length(b.center - a.center) <= 1e-8f);
        const float ax[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        float best = 3.402823466e38f;
        f3 best_normal = mk3(0.0f, 1.0f, 0.0f);
        for (uint32_t k = 0; k < kProbeEnd; ++k) {
            f3 d;
            if (k < kProbeCentre) {
                if (!(triples & (1u << k))) continue;
                const f3 wi = sw[kProbeTriple[k][0]], wj = sw[kProbeTriple[k][1]], wk = sw[kProbeTriple[k][2]];
                d = normalize(cross(wj - wi, wk - wi));
            } else if (k == kProbeCentre) {
                if (!centre) continue;
                d = normalize(b.center - a.center);
            } else {
                const uint32_t x = k - kProbeAxes;
                d = normalize(mk3(ax[x][0], ax[x][1], ax[x][2]));
            }
            const SPt sp = support_pair(w, a, b, d);
            const float depth = dot(sp.w, d);
            if (depth < best) {
                best = depth;
                best_normal = d;
            }
            if (depth <= 0.0f) break;
        }
        Hit hit{3.402823466e38f, s3(0.0f), s3(0.0f)};
        if (best > 0.0f) {
            f3 nrm = best_normal;
            if (dot(nrm, b.center - a.center) < 0.0f) nrm = -nrm;
            hit = Hit{-best, (pa + pb) * 0.5f, nrm};
        } else if (dist > 0.0f) {
            hit = Hit{dist, (pa + pb) * 0.5f, normal};
        }
        if (hit.distance <= margin) push_hit(w, index, hit);
    }
}

// Phase 2: one lane group (half a warp) per penetrating pair: the polytopes of this path hold a few
// dozen faces, which sixteen lanes cover in one or two strides, so two pairs share each warp's
// instructions.
constexpr int kEpaWarpsPerBlock = 4;
constexpr uint32_t kEpaLanes = 16;
constexpr uint32_t kEpaGroupsPerBlock = kEpaWarpsPerBlock * (32u / kEpaLanes);
__global__ void __launch_bounds__(32 * kEpaWarpsPerBlock) k_convex_epa(DeviceWorld w, dyn_step_params p) {
    __shared__ EpaWarpShared shared[kEpaGroupsPerBlock];
    const uint32_t count = min(w.ctl[CTL_EPA], w.p_cap);
    const Lanes<kEpaLanes> L;
    const uint32_t group = threadIdx.x / kEpaLanes;
    EpaWarpShared& m = shared[group];
    for (;;) {  // each lane group takes the next pair from a shared ticket: pairs differ in cost
        uint32_t e = 0u;
        if (L.lane == 0u) e = atomicAdd(&w.ctl[CTL_EPA_NEXT], 1u);
        e = L.shfl(e, 0u);
        if (e >= count) break;
        uint32_t index = w.epa_list[e];
        WShape a, b;
        DBody fb, sb;
        convex_shapes(w, index, &a, &b, &fb, &sb);
        f3 simplex[4];
        for (uint32_t k = 0; k < 4; ++k) simplex[k] = xyz(w.epa_simplex[4 * (size_t)e + k]);
        Hit hit = warp_penetrating_hit(L, w, a, b, simplex, m);
        if (L.lane == 0u) {
            if (hit.distance <= pair_margin(p, fb, sb)) push_hit(w, index, hit);
        }
        L.sync();
    }
}

// Phase 3: the feature-ring manifold for every hit (convex_pair_manifold, else manifold_from_hit).
__global__ void __launch_bounds__(128) k_convex_manifold(DeviceWorld w, dyn_step_params p) {
    const uint32_t count = min(w.ctl[CTL_HITS], w.p_cap);
    GRID_STRIDE(i, count) {
        uint32_t index = w.hit_list[i];
        float4 h0 = w.hit_data[2 * (size_t)i], h1 = w.hit_data[2 * (size_t)i + 1];
        uint32_t fs = w.pmaj[index], ss = w.pmin[index];
        uint32_t fr = w.c_owner[fs], sr = w.c_owner[ss];
        DBody fb = load_dbody(w.hot, fr), sb = load_dbody(w.hot, sr);
        DColl fc = load_dcoll(w, fs), sc = load_dcoll(w, ss);
        WShape a = world_shape(fb.position, fb.orientation, fc);
        WShape b = world_shape(sb.position, sb.orientation, sc);
        float margin = pair_margin(p, fb, sb);
        Mani m;
        mani_emit(&m, xyz(h1));
        if (!convex_pair_manifold(w, a, b, xyz(h1), &m)) {
            if (h0.w <= margin) mani_push(&m, xyz(h0), -h0.w, kFeatPoint);
        }
        if (m.count > 0u) {
            uint32_t slot = append_slot(&w.ctl[CTL_APPENDED]);
            if (slot < w.s_cap) {
                uint4 fi = w.ident[fr], si = w.ident[sr];
                bool sensor = (fc.flags & DYN_COLLIDER_SENSOR) != 0u || (sc.flags & DYN_COLLIDER_SENSOR) != 0u;
                write_contact(w.tmp, w.s_cap, slot, m, fr, sr, fs, ss, fb, sb, fi.x, si.x, fi.y, si.y, sensor, w.c_mat[fs],
                              w.c_mat[ss], w.c_mat2[fs], w.c_mat2[ss], fc.flags, sc.flags, p.friction_combine,
                              p.restitution_combine);
            } else {
                add_counter(&w.counters[DYN_COUNTER_REFUSED_CONTACTS], 1u);
            }
        }
    }
}

// Four blocks per SM: the analytic class then holds 128 registers (a few spilled) instead of 168,
// which measured faster than the three blocks its registers allow otherwise.
template <int kClass>
__global__ void __launch_bounds__(128, 4) k_narrow_class(DeviceWorld w, dyn_step_params p) {
    const uint32_t count = min(w.ctl[CTL_LIST0 + kClass], w.p_cap);
    const uint32_t* list = w.np_list + (size_t)kClass * w.p_cap;
    GRID_STRIDE(i, count) narrow_pair<kClass>(w, p, list[i]);
}

// ---- compaction (compact_scan.wgsl, compact_offsets.wgsl, compact_scatter.wgsl) ----
// The reference sorts all candidate pairs and compacts the narrowphase output in pair order. Here
// the pairs stay in emission order; the narrowphase appends its contacts to a staging set as large
// as the pair stream (a pair yields at most one contact, so every contact found is staged), the
// staged contacts alone are sorted by (lower, higher) collider slot, and the first c_cap of them in
// that order are gathered: the contacts and the ones refused past the capacity are the reference's
// (compact_scatter.wgsl keeps the first in pair order), whatever order the narrowphase finished in.
__global__ void k_contact_keys(DeviceWorld w) {
    const uint32_t appended = w.ctl[CTL_APPENDED];
    const uint32_t staged = min(appended, w.s_cap);
    const uint32_t c = min(staged, w.c_cap);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        w.counters[DYN_COUNTER_CONTACTS] = c;
        w.ctl[CTL_STAGED] = staged;
        w.ctl[CTL_CONTACTS] = c;
        w.counters[DYN_COUNTER_BLOCKS] = c;
        if (staged > c) w.counters[DYN_COUNTER_REFUSED_CONTACTS] += staged - c;
    }
    GRID_STRIDE(i, staged) {
        const uint4 ids = w.tmp.ids[i];
        w.cmaj[i] = ids.x;
        w.cmin[i] = ids.y;
        w.cval[i] = i;
    }
}
__device__ __forceinline__ void copy_contact(const ContactSet& from, uint32_t fi, uint32_t from_cap, const ContactSet& to,
                                             uint32_t ti, uint32_t cap) {
    uint4 rows = from.rows[fi];
    to.normal[ti] = from.normal[fi];
    to.rows[ti] = rows;
    to.mat[ti] = from.mat[fi];
    to.ids[ti] = from.ids[fi];
    to.ids2[ti] = from.ids2[fi];
    to.extra[ti] = from.extra[fi];
    uint32_t count = rows.z & 0xFFu;
    for (uint32_t p = 0; p < count; ++p) {
        size_t f = (size_t)p * from_cap + fi, t = (size_t)p * cap + ti;
        to.la[t] = from.la[f];
        to.lb[t] = from.lb[f];
        to.acc[t] = from.acc[f];
        to.pos[t] = from.pos[f];
    }
}
__global__ void k_contact_gather(DeviceWorld w) {
    const uint32_t c = w.ctl[CTL_CONTACTS];
    GRID_STRIDE(i, c) {
        copy_contact(w.tmp, w.cval[i], w.s_cap, w.cur, i, w.c_cap);
        w.matched[i] = 0u;
    }
}

// ---- warm-start identity (identity.wgsl, contact_relay.wgsl, contact_begin.wgsl) ----
__device__ __forceinline__ bool same_pair(uint4 hi, uint4 hi2, uint4 ci, uint4 ci2) {
    bool same = hi.z == ci.z && hi2.x == ci2.x && hi.w == ci.w && hi2.y == ci2.y && hi.x == ci.x && hi.y == ci.y;
    bool flipped = hi.z == ci.w && hi2.x == ci2.y && hi.w == ci.z && hi2.y == ci2.x && hi.x == ci.y && hi.y == ci.x;
    return same || flipped;
}
__device__ __forceinline__ uint32_t resolve_row(const DeviceWorld& w, uint32_t id, uint32_t gen) {
    if (id >= w.id_count) return DYN_NO_BODY;
    uint32_t row = w.row_of_id[id];
    if (row == DYN_NO_BODY || w.ident[row].y != gen) return DYN_NO_BODY;
    return row;
}
__device__ __forceinline__ bool touches(const ContactSet& s, uint32_t i, uint32_t cap, float threshold) {
    uint32_t count = s.rows[i].z & 0xFFu;
    for (uint32_t p = 0; p < count; ++p) {
        if (s.la[(size_t)p * cap + i].w >= -threshold) return true;
    }
    return false;
}

// contact_relay.wgsl:34-71 over last step's contacts.
__global__ void k_relay(DeviceWorld w) {
    const uint32_t held_n = w.ctl[CTL_ARCHIVED];
    const uint32_t count = w.ctl[CTL_CONTACTS];
    const uint32_t cap = w.c_cap;
    GRID_STRIDE(h, held_n) {
        uint4 hi = w.arc.ids[h], hi2 = w.arc.ids2[h];
        uint4 hrows = w.arc.rows[h];
        if (resolve_row(w, hi.z, hi2.x) == DYN_NO_BODY || resolve_row(w, hi.w, hi2.y) == DYN_NO_BODY) continue;
        uint32_t lo = 0, hi_ = count;
        while (lo < hi_) {
            uint32_t mid = (lo + hi_) >> 1;
            uint4 c = w.cur.ids[mid];
            if (c.x < hi.x || (c.x == hi.x && c.y < hi.y)) lo = mid + 1;
            else hi_ = mid;
        }
        if (!(lo < count)) continue;
        uint4 ci = w.cur.ids[lo];
        if (!(ci.x == hi.x && ci.y == hi.y)) continue;
        uint4 ci2 = w.cur.ids2[lo];
        if (!same_pair(hi, hi2, ci, ci2)) continue;
        if ((hrows.w & DYN_CONTACT_ANNOUNCED) == 0u) continue;
        w.matched[lo] = 1u;
        uint4 crows = w.cur.rows[lo];
        uint32_t ccount = crows.z & 0xFFu, hcount = hrows.z & 0xFFu;
        bool taken[4] = {false, false, false, false};
        float carried_n = 0.0f, carried_t = 0.0f;
        for (uint32_t pi = 0; pi < ccount; ++pi) {
            size_t co = (size_t)pi * cap + lo;
            float4 cacc = w.cur.acc[co];
            uint32_t feature = __float_as_uint(cacc.w);
            f3 cla = xyz(w.cur.la[co]), clb = xyz(w.cur.lb[co]);
            uint32_t picked = DYN_NO_SLOT;
            float picked_d = 0.0f;
            for (uint32_t hj = 0; hj < hcount; ++hj) {
                if (taken[hj]) continue;
                size_t ho = (size_t)hj * cap + h;
                uint32_t hf = __float_as_uint(w.arc.acc[ho].w);
                if (!(hf == feature || hf == feature_mirror(feature))) continue;
                float d = length(xyz(w.arc.la[ho]) - cla) + length(xyz(w.arc.lb[ho]) - clb);
                if (picked == DYN_NO_SLOT || d < picked_d) {
                    picked = hj;
                    picked_d = d;
                }
            }
            float4 nacc = cacc;
            if (picked != DYN_NO_SLOT) {
                taken[picked] = true;
                if (w.tape.relay) w.tape.relay[(size_t)(*w.tape.slot) * 4u * cap + co] = picked * cap + h;
                float4 hacc = w.arc.acc[(size_t)picked * cap + h];
                nacc = make_float4(hacc.x, hacc.y, hacc.z, cacc.w);
                w.cur.acc[co] = nacc;
            }
            carried_n = carried_n + wmax(nacc.x, 0.0f);
            carried_t = carried_t + sqrtf(nacc.y * nacc.y + nacc.z * nacc.z);
        }
        float4 ex = w.cur.extra[lo];
        w.cur.extra[lo] = make_float4(ex.x, carried_n, carried_t, 0.0f);
        w.cur.rows[lo] = make_uint4(crows.x, crows.y, crows.z, crows.w | DYN_CONTACT_ANNOUNCED);
    }
}

// contact_begin.wgsl:41-71 (the resting index, which only decides event announcements, is not
// consulted): unmatched touching contacts are announced.
__global__ void k_contact_begin(DeviceWorld w, dyn_step_params p) {
    const uint32_t count = w.ctl[CTL_CONTACTS];
    GRID_STRIDE(i, count) {
        if (w.matched[i] != 0u) continue;
        if (touches(w.cur, i, w.c_cap, p.slop)) {
            uint4 r = w.cur.rows[i];
            w.cur.rows[i] = make_uint4(r.x, r.y, r.z, r.w | DYN_CONTACT_ANNOUNCED);
        }
    }
}

// ---- islands (island_link*.wgsl, island_flatten.wgsl, island_aggregate.wgsl, island_count.wgsl) ----
// Union-find over the dynamic rows, hooking the higher root under the lower one, so each island's
// root is its smallest row. Parents are read with ld.global.cg: the L2 copy every CAS acts on (an L1
// copy could stay stale for the whole kernel). Finding halves the path: a non-root row's parent
// entry only ever moves to one of its own ancestors, and roots change only through the CAS, so the
// plain store of the grandparent never undoes a hook.
__device__ __forceinline__ uint32_t island_find(const DeviceWorld& w, uint32_t node) {
    uint32_t current = node;
    uint32_t parent = __ldcg(w.parents + current);
    for (uint32_t guard = 0; parent != current && guard < w.nd; ++guard) {
        uint32_t grand = __ldcg(w.parents + parent);
        if (grand != parent) w.parents[current] = grand;
        current = grand;
        parent = __ldcg(w.parents + current);
    }
    return current;
}
// island_couple (island_link.wgsl:3-45): a static row carries its wake flag to the other row, and
// two dynamic rows join one island. The union returns false when its bounded retries gave up.
__device__ __forceinline__ void island_carry(const DeviceWorld& w, uint32_t first, uint32_t second) {
    uint32_t dc = w.nd;
    if (second >= dc && w.wake_flags[second] != 0u) atomicOr(&w.wake_flags[first], 1u);
    if (first >= dc && w.wake_flags[first] != 0u) atomicOr(&w.wake_flags[second], 1u);
}
__device__ __forceinline__ bool island_union(const DeviceWorld& w, uint32_t first, uint32_t second) {
    uint32_t dc = w.nd;
    if (first >= dc || second >= dc || first == second) return true;
    for (uint32_t attempt = 0; attempt < 256u; ++attempt) {
        uint32_t a = island_find(w, first), b = island_find(w, second);
        if (a == b) return true;
        uint32_t lower = min(a, b), higher = max(a, b);
        if (atomicCAS(&w.parents[higher], higher, lower) == higher) return true;
    }
    return false;
}
__device__ __forceinline__ bool island_couple(const DeviceWorld& w, uint32_t first, uint32_t second) {
    island_carry(w, first, second);
    return island_union(w, first, second);
}
// The contacts join islands in two passes with a flatten between (the sampling idea of Afforest,
// Sutton et al. 2018): first only the first contact of each collider's run in the sorted list,
// which already ties most of a pile together; after the flatten every row points at its root, so
// a later contact whose rows share a parent is skipped without a find. Which contact hooks which
// root does not change the islands, and each island's root stays its smallest row.
template <bool kSample>
__global__ void k_island_link(DeviceWorld w, dyn_step_params p) {
    const uint32_t count = w.ctl[CTL_CONTACTS];
    GRID_STRIDE(i, count) {
        uint4 r = w.cur.rows[i];
        uint32_t pc = r.z & 0xFFu, sensor = (r.z >> 8) & 0xFFu;
        if (pc == 0u || sensor == 1u || !touches(w.cur, i, w.c_cap, p.slop)) continue;
        const bool first_of_run = i == 0u || w.cur.ids[i - 1u].x != w.cur.ids[i].x;
        if (kSample) {
            island_carry(w, r.x, r.y);
            if (!first_of_run) continue;
        } else {
            if (first_of_run) continue;
            if (r.x < w.nd && r.y < w.nd && __ldcg(w.parents + r.x) == __ldcg(w.parents + r.y)) continue;
        }
        if (!island_union(w, r.x, r.y)) add_counter(&w.counters[DYN_COUNTER_ISLAND_FAULTS], 1u);
    }
    if (kSample) return;
    // island_link_resting.wgsl:10-21 in the same pass: every frozen contact (rest.cuh) couples its
    // two rows; unions commute, so sharing the launch with the contacts changes no island
    const uint32_t frozen = min(w.ctl[CTL_RESTING], w.rest_cap);
    GRID_STRIDE(i, frozen) {
        const uint4 r = w.rest_in[i];
        const uint32_t a = resolve_row(w, r.x, r.y), b = resolve_row(w, r.z, r.w);
        if (a == DYN_NO_BODY || b == DYN_NO_BODY) continue;
        if (!island_couple(w, a, b)) add_counter(&w.counters[DYN_COUNTER_ISLAND_FAULTS], 1u);
    }
}
// island_flatten.wgsl:4-8 repeated ilog2(max(N,2))+1 times leaves every row pointing at its root
// (pointer jumping doubles the reach each round and a chain is at most N long); one pass that
// follows each chain to its root gives that same array. Roots no longer change here, and rows
// rewritten concurrently only ever point further up their own chain.
// After the last links (kAggregate) the root each row finds is final, so the same pass does
// island_aggregate's work (island_aggregate.wgsl): count the islands and mark the ones to wake.
template <bool kAggregate>
__global__ void k_island_flatten(DeviceWorld w) {
    GRID_STRIDE(i, w.nd) {
        uint32_t root = i;
        uint32_t parent = __ldcg(w.parents + root);
        for (uint32_t guard = 0; parent != root && guard < w.nd; ++guard) {
            root = parent;
            parent = __ldcg(w.parents + root);
        }
        w.parents[i] = root;
        if (!kAggregate) continue;
        if (root == i) add_counter(&w.counters[DYN_COUNTER_ISLANDS], 1u);
        if (w.wake_flags[i] == 0u && w.motion[i] == 0u) continue;
        if (__ldcg(w.istate + root) >= DYN_ISLAND_WAKE) continue;
        atomicMax(&w.istate[root], DYN_ISLAND_WAKE);
    }
}
// island_wake.wgsl:10-22 then live.wgsl:8-18 for the same row.
__global__ void k_wake_live(DeviceWorld w) {
    GRID_STRIDE(i, w.nd) {
        uint32_t root = w.parents[i];
        BodyHot& h = w.hot[i];
        uint32_t sleeping = h.aux.x;
        if (sleeping != 0u && (w.istate[root] & DYN_ISLAND_WAKE) != 0u) {
            add_counter(&w.counters[DYN_COUNTER_WOKE], 1u);
            add_counter(&w.counters[DYN_COUNTER_WOKE_DEFERRED], 1u);
            h.aux.x = 0u;
            sleeping = 0u;
            w.sleep_timer[i] = 0.0f;
        }
        w.wake_flags[i] = 0u;
        if (moves(h.pos.w, h.aux.y) && sleeping == 0u) {
            uint32_t slot = append_slot(&w.ctl[CTL_LIVE]);
            w.live[slot] = i;
        }
    }
}

// ---- solver (solver_blocks.wgsl, solver_contact_block.wgsl, solver_block_apply.wgsl) ----
__device__ __forceinline__ bool resolves(uint4 rows) { return (rows.z & 0xFFu) > 0u && ((rows.z >> 8) & 0xFFu) == 0u; }

__global__ void k_solver_blocks(DeviceWorld w, dyn_step_params p) {
    const uint32_t count = w.ctl[CTL_CONTACTS];
    const uint32_t cap = w.c_cap;
    GRID_STRIDE(i, count) {
        uint4 r = w.cur.rows[i];
        if (!resolves(r)) {
            w.cowner[i] = 0u;
            continue;
        }
        DBody fb = load_dbody(w.hot, r.x), sb = load_dbody(w.hot, r.y);
        f3 normal = xyz(w.cur.normal[i]);
        float restitution = w.cur.extra[i].x;
        uint32_t pc = r.z & 0xFFu;
        for (uint32_t pi = 0; pi < pc; ++pi) {
            size_t o = (size_t)pi * cap + i;
            f3 position = xyz(w.cur.pos[o]);
            float depth = w.cur.la[o].w;
            float speed = dot(relative_velocity(fb, sb, position, position), normal);
            float target = 0.0f;
            if (depth < 0.0f) {
                target = depth / p.dt;
            } else if (speed < -p.restitution_threshold) {
                target = -speed * restitution;
            }
            float4 lb = w.cur.lb[o];
            w.cur.lb[o] = make_float4(lb.x, lb.y, lb.z, target);
        }
        uint32_t own = 0u;
        if (atomicAdd(&w.hot[r.x].aux.z, 1u) == 0u) {
            w.row_flag[r.x] = 1u;
            own |= 1u;
        }
        if (atomicAdd(&w.hot[r.y].aux.z, 1u) == 0u) {
            w.row_flag[r.y] = 1u;
            own |= 2u;
        }
        w.cowner[i] = own;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) w.counters[DYN_COUNTER_BLOCKS] = count;
}
// The claimed rows in ascending order (scanned flags): the applies then walk the body rows in
// memory order instead of claim order. The set of rows is the reference's; their order changes
// nothing, each row being applied on its own.
__global__ void k_solver_row_list(DeviceWorld w) {
    GRID_STRIDE(i, w.n) {
        if (w.row_flag[i] != 0u) w.solver_rows[w.row_offset[i]] = i;
    }
}

__device__ __forceinline__ int32_t solver_word(float value, float scale) { return (int32_t)wclamp(value * scale, -2.0e9f, 2.0e9f); }
__device__ __forceinline__ void accumulate(int32_t* deltas, uint32_t row, f3 lin, f3 ang, float scale) {
    int32_t* d = deltas + 8u * row;
    atomicAdd(d + 0, solver_word(lin.x, scale));
    atomicAdd(d + 1, solver_word(lin.y, scale));
    atomicAdd(d + 2, solver_word(lin.z, scale));
    atomicAdd(d + 3, solver_word(ang.x, scale));
    atomicAdd(d + 4, solver_word(ang.y, scale));
    atomicAdd(d + 5, solver_word(ang.z, scale));
}
// The linear words alone: position corrections carry no angular part, and adding a zero word
// changes nothing, so the three angular atomics are left out.
__device__ __forceinline__ void accumulate_linear(int32_t* deltas, uint32_t row, f3 lin, float scale) {
    int32_t* d = deltas + 8u * row;
    atomicAdd(d + 0, solver_word(lin.x, scale));
    atomicAdd(d + 1, solver_word(lin.y, scale));
    atomicAdd(d + 2, solver_word(lin.z, scale));
}
__device__ __forceinline__ void make_tangents(f3 n, f3* t1, f3* t2) {
    f3 t = fabsf(n.x) > 0.9f ? mk3(0.0f, 1.0f, 0.0f) : mk3(1.0f, 0.0f, 0.0f);
    *t1 = normalize(cross(n, t));
    *t2 = cross(n, *t1);
}
__device__ __forceinline__ f3 arm(const DBody& b, f3 local) { return quat_rotate(b.orientation, local) + b.position; }
__device__ __forceinline__ void pair_impulse(DBody* a, DBody* b, f3 pa, f3 pb, f3 j) {
    a->velocity = a->velocity - j * a->inverse_mass;
    a->angular_velocity = a->angular_velocity - dbody_iinv(*a, cross(pa - dbody_com(*a), j));
    b->velocity = b->velocity + j * b->inverse_mass;
    b->angular_velocity = b->angular_velocity + dbody_iinv(*b, cross(pb - dbody_com(*b), j));
}
__device__ __forceinline__ float momentum_mass(const DBody& a, const DBody& b, f3 pa, f3 pb, f3 axis) {
    f3 ra = pa - dbody_com(a), rb = pb - dbody_com(b);
    f3 rax = cross(ra, axis), rbx = cross(rb, axis);
    return a.inverse_mass + b.inverse_mass + dot(rax, dbody_iinv(a, rax)) + dot(rbx, dbody_iinv(b, rbx));
}
__device__ __forceinline__ DBody split_body(DBody b, float s) {
    b.inverse_mass = b.inverse_mass * s;
    b.ii0 = make_float4(b.ii0.x * s, b.ii0.y * s, b.ii0.z * s, b.ii0.w * s);
    b.ii1 = make_float2(b.ii1.x * s, b.ii1.y * s);
    return b;
}

// ---- pose-only terms of each contact block, once per substep ----
// Between integrate and advance no pose changes, so the contact arms, the effective masses along
// the normal and both tangents and the twist mass are the same in the warm start and in every
// velocity iteration of a substep. k_solve_prepare computes them once per substep with the very
// expressions solver_contact_block.wgsl:24-80 uses (stored floats reload bit for bit), and k_warm
// and k_solve read them. arm_a/arm_b hold a contact point minus the body's world centre of mass,
// the operand that point_velocity and the impulse torques take.
__device__ __forceinline__ f3 point_velocity_arm(const DBody& b, f3 arm_from_com) {
    return b.velocity + cross(b.angular_velocity, arm_from_com);
}
__device__ __forceinline__ void pair_impulse_arms(DBody* a, DBody* b, f3 ra, f3 rb, f3 j) {
    a->velocity = a->velocity - j * a->inverse_mass;
    a->angular_velocity = a->angular_velocity - dbody_iinv(*a, cross(ra, j));
    b->velocity = b->velocity + j * b->inverse_mass;
    b->angular_velocity = b->angular_velocity + dbody_iinv(*b, cross(rb, j));
}
__device__ __forceinline__ float momentum_mass_arms(const DBody& a, const DBody& b, f3 ra, f3 rb, f3 axis) {
    f3 rax = cross(ra, axis), rbx = cross(rb, axis);
    return a.inverse_mass + b.inverse_mass + dot(rax, dbody_iinv(a, rax)) + dot(rbx, dbody_iinv(b, rbx));
}
// The two bodies of a contact as the block sees them: the bodies, their mass-split copies, and the
// frozen (massless) form of an inert one.
struct BlockBodies {
    DBody pf, ps, sf, ss;
};
__device__ __forceinline__ BlockBodies block_bodies(const DeviceWorld& w, uint4 r) {
    BlockBodies b;
    b.pf = load_dbody(w.hot, r.x);
    b.ps = load_dbody(w.hot, r.y);
    b.sf = split_body(b.pf, (float)max(w.hot[r.x].aux.z, 1u));
    b.ss = split_body(b.ps, (float)max(w.hot[r.y].aux.z, 1u));
    if (dbody_inert(b.pf)) {
        b.pf = dbody_frozen(b.pf);
        b.sf = dbody_frozen(b.sf);
    }
    if (dbody_inert(b.ps)) {
        b.ps = dbody_frozen(b.ps);
        b.ss = dbody_frozen(b.ss);
    }
    return b;
}

// The row-mass guard (DYN_SOLVER_GUARD_ROW_MASS, no counterpart in the reference). A block solves
// its points' normal rows Jacobi-wise against the manifold row masses D_j = sum_k A_jk
// (manifold_row_mass, solver_contact_block.wgsl:14-29), A being the points' coupling matrix
// A_jk = m_a + m_b + (r_aj x n) . I_a (r_ak x n) + (r_bj x n) . I_b (r_bk x n) of the split bodies.
// The iteration converges while the eigenvalues of S = D^-1/2 A D^-1/2 stay below 2; where a point's
// arm opposes the others' (a tilted box landing on three points) they do not, and the impulses grow
// twofold or more per iteration. The guard keeps a block's row masses when every D_j is positive
// and kRowMassBound I - S is positive definite (its LDL^T pivots all positive), i.e. every
// eigenvalue of S lies below kRowMassBound; otherwise each point takes count x A_jj, whose
// normalised matrix has unit diagonal and off-diagonal entries within 1, so its eigenvalues stay
// at or below count / count = 1.
constexpr float kRowMassBound = 1.9f;
__device__ __forceinline__ float coupling(const DBody& a, const DBody& b, f3 uj, f3 vj, f3 iuk, f3 ivk) {
    return a.inverse_mass + b.inverse_mass + dot(uj, iuk) + dot(vj, ivk);
}
__device__ __forceinline__ void guard_row_masses(const BlockBodies& b, f3 normal, const f3* ra, const f3* rb, uint32_t pc,
                                                 float count_f, float* nm) {
    f3 u[4], v[4], iu[4], iv[4];
    for (uint32_t j = 0; j < pc; ++j) {
        u[j] = cross(ra[j], normal);
        v[j] = cross(rb[j], normal);
        iu[j] = dbody_iinv(b.sf, u[j]);
        iv[j] = dbody_iinv(b.ss, v[j]);
    }
    bool converges = true;
    for (uint32_t j = 0; j < pc; ++j) converges = converges && nm[j] > 0.0f;
    if (converges) {
        // M = bound I - S, factored M = L diag(d) L^T row by row
        float m[4][4], l[4][4], d[4];
        for (uint32_t j = 0; j < pc; ++j)
            for (uint32_t k = 0; k < pc; ++k)
                m[j][k] = (j == k ? kRowMassBound : 0.0f) - coupling(b.sf, b.ss, u[j], v[j], iu[k], iv[k]) / sqrtf(nm[j] * nm[k]);
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
    if (converges) return;
    for (uint32_t j = 0; j < pc; ++j) nm[j] = count_f * coupling(b.sf, b.ss, u[j], v[j], iu[j], iv[j]);
}

__global__ void k_solve_prepare(DeviceWorld w) {
    const uint32_t count = w.ctl[CTL_CONTACTS];
    const uint32_t cap = w.c_cap;
    const SolverRows& sr = w.srows;
    GRID_STRIDE(i, count) {
        uint4 r = w.cur.rows[i];
        if (!resolves(r)) continue;
        const BlockBodies b = block_bodies(w, r);
        if (dbody_inert(b.pf) && dbody_inert(b.ps)) continue;
        f3 normal = xyz(w.cur.normal[i]);
        f3 t1, t2;
        make_tangents(normal, &t1, &t2);
        uint32_t pc = r.z & 0xFFu;
        f3 ra[4], rb[4];
        f3 reach_f = s3(0.0f), reach_s = s3(0.0f);
        for (uint32_t pi = 0; pi < pc; ++pi) {
            size_t o = (size_t)pi * cap + i;
            f3 af = arm(b.pf, xyz(w.cur.la[o]));
            f3 as = arm(b.ps, xyz(w.cur.lb[o]));
            ra[pi] = af - dbody_com(b.pf);
            rb[pi] = as - dbody_com(b.ps);
            reach_f = reach_f + ra[pi];
            reach_s = reach_s + rb[pi];
        }
        float count_f = (float)max(pc, 1u);
        f3 spread_f = dbody_iinv(b.sf, cross(reach_f, normal));
        f3 spread_s = dbody_iinv(b.ss, cross(reach_s, normal));
        float nm[4];
        for (uint32_t pi = 0; pi < pc; ++pi) {
            f3 arm_f = cross(ra[pi], normal);
            f3 arm_s = cross(rb[pi], normal);
            nm[pi] = count_f * (b.sf.inverse_mass + b.ss.inverse_mass) + dot(spread_f, arm_f) + dot(spread_s, arm_s);
        }
        if ((w.solver_guard & DYN_SOLVER_GUARD_ROW_MASS) && pc >= 2u) guard_row_masses(b, normal, ra, rb, pc, count_f, nm);
        for (uint32_t pi = 0; pi < pc; ++pi) {
            size_t o = (size_t)pi * cap + i;
            float normal_mass = nm[pi];
            float truth = momentum_mass_arms(b.pf, b.ps, ra[pi], rb[pi], normal);
            float t1_mass = momentum_mass_arms(b.sf, b.ss, ra[pi], rb[pi], t1) * count_f;
            float t2_mass = momentum_mass_arms(b.sf, b.ss, ra[pi], rb[pi], t2) * count_f;
            sr.arm_a[o] = mk4(ra[pi], normal_mass);
            sr.arm_b[o] = mk4(rb[pi], truth);
            sr.masses[o] = make_float4(t1_mass, t2_mass, w.cur.la[o].w, w.cur.lb[o].w);
        }
        float twist_mass = dot(normal, dbody_iinv(b.sf, normal)) + dot(normal, dbody_iinv(b.ss, normal));
        sr.tangent1[i] = mk4(t1, twist_mass);
        sr.tangent2[i] = mk4(t2, 0.0f);
    }
}

// solver_contact_block.wgsl:195-233
__global__ void k_warm(DeviceWorld w) {
    const uint32_t count = w.ctl[CTL_CONTACTS];
    const uint32_t cap = w.c_cap;
    const SolverRows& sr = w.srows;
    GRID_STRIDE(i, count) {
        uint4 r = w.cur.rows[i];
        if (!resolves(r)) continue;  // zero deltas change nothing
        DBody fl = load_dbody(w.hot, r.x), sl = load_dbody(w.hot, r.y);
        DBody f = dbody_inert(fl) ? dbody_frozen(fl) : fl;
        DBody s = dbody_inert(sl) ? dbody_frozen(sl) : sl;
        if (dbody_inert(fl) && dbody_inert(sl)) continue;  // no rows were prepared; both deltas are zero
        f3 normal = xyz(w.cur.normal[i]);
        f3 t1 = xyz(sr.tangent1[i]), t2 = xyz(sr.tangent2[i]);
        uint32_t pc = r.z & 0xFFu;
        for (uint32_t pi = 0; pi < pc; ++pi) {
            size_t o = (size_t)pi * cap + i;
            float4 acc = w.cur.acc[o];
            f3 j = normal * acc.x + t1 * acc.y + t2 * acc.z;
            pair_impulse_arms(&f, &s, xyz(sr.arm_a[o]), xyz(sr.arm_b[o]), j);
        }
        // an inert (frozen) body's delta is exactly zero: its atomics would add nothing
        if (!dbody_inert(fl))
            accumulate(w.vdelta, r.x, f.velocity - fl.velocity, f.angular_velocity - fl.angular_velocity, DYN_SOLVER_VELOCITY_SCALE);
        if (!dbody_inert(sl))
            accumulate(w.vdelta, r.y, s.velocity - sl.velocity, s.angular_velocity - sl.angular_velocity, DYN_SOLVER_VELOCITY_SCALE);
    }
}

// solver_contact_block.wgsl:6-193 (Jacobi block with mass splitting); the pose-only terms come
// from k_solve_prepare.
__device__ __forceinline__ void solve_block(const DeviceWorld& w, const dyn_step_params& p, uint32_t i, bool residual,
                                            uint32_t tape_index) {
    const uint32_t cap = w.c_cap;
    const SolverRows& sr = w.srows;
    uint4 r = w.cur.rows[i];
    if (!resolves(r)) return;
    const BlockBodies b = block_bodies(w, r);
    const DBody& pf = b.pf;
    const DBody& ps = b.ps;
    if (dbody_inert(pf) && dbody_inert(ps)) return;
    float4* tape_acc = nullptr;
    if (w.tape.vel) {
        // a taped step: the velocities and impulses this iteration starts from (every block of a
        // row writes the same velocities)
        const TapeWrites& t = w.tape;
        const size_t slot = *t.slot;
        float4* vel = t.vel + (slot * t.substeps * t.iterations + tape_index) * 2 * t.n;
        vel[r.x] = w.hot[r.x].vel;
        vel[t.n + r.x] = w.hot[r.x].ang;
        vel[r.y] = w.hot[r.y].vel;
        vel[t.n + r.y] = w.hot[r.y].ang;
        tape_acc = t.acc + (slot * t.substeps * t.iterations + tape_index) * 4 * t.c;
    }
    DBody first = pf, second = ps;
    float4 nf = w.cur.normal[i];
    f3 normal = xyz(nf);
    float friction = nf.w;
    float4 mat = w.cur.mat[i];
    float4 tw1 = sr.tangent1[i];
    f3 t1 = xyz(tw1), t2 = xyz(sr.tangent2[i]);
    float twist_mass = tw1.w;
    uint32_t pc = r.z & 0xFFu;
    // One point at a time: every point's impulse is computed from the velocities the block started
    // with (pf, ps), so applying each to first/second as soon as it is known gives the same sums,
    // in the same order, as applying all four after the loop; the old normal accumulators are summed
    // in point order as they are read. Only one point's data is live at a time.
    float normal_total = 0.0f;
    #pragma unroll
    for (uint32_t pi = 0; pi < 4u; ++pi) if (pi < pc) {
        size_t o = (size_t)pi * cap + i;
        float4 acc = w.cur.acc[o];
        if (tape_acc) tape_acc[(size_t)pi * w.tape.c + i] = acc;
        normal_total = normal_total + wmax(acc.x, 0.0f);
        float4 a4 = sr.arm_a[o], b4 = sr.arm_b[o];
        float4 m2 = sr.masses[o];
        const f3 ra = xyz(a4), rb = xyz(b4);
        float normal_mass = a4.w, truth = b4.w;
        float depth = m2.z, target = m2.w;
        float an = acc.x, at1 = acc.y, at2 = acc.z;
        f3 rel = point_velocity_arm(ps, rb) - point_velocity_arm(pf, ra);
        float normal_speed = dot(rel, normal);
        float delta;
        if (mat.z <= 0.0f) {
            delta = (target - normal_speed) / normal_mass;
        } else {
            float bias = wmax(depth / p.dt, target);
            float drag = 2.0f * mat.w * mat.z / p.dt;
            float softness = mat.z * mat.z * truth / (p.dt * p.dt);
            float prior = normal_speed - an * truth;
            float wanted = (bias - (1.0f + drag) * prior) / (softness + (1.0f + drag) * truth);
            delta = truth * (wanted - an) / normal_mass;
        }
        float next_n = wmax(0.0f, an + delta);
        f3 impulse = s3(0.0f) + normal * (next_n - an);
        an = next_n;
        float limit = friction * an;
        float t1_speed = dot(rel, t1);
        float next_t1 = wclamp(at1 - t1_speed / m2.x, -limit, limit);
        impulse = impulse + t1 * (next_t1 - at1);
        at1 = next_t1;
        float t2_speed = dot(rel, t2);
        float remaining = sqrtf(wmax(limit * limit - at1 * at1, 0.0f));
        float next_t2 = wclamp(at2 - t2_speed / m2.y, -remaining, remaining);
        impulse = impulse + t2 * (next_t2 - at2);
        at2 = next_t2;
        w.cur.acc[o] = make_float4(an, at1, at2, acc.w);
        pair_impulse_arms(&first, &second, ra, rb, impulse);
    }
    f3 rel_spin = second.angular_velocity - first.angular_velocity;
    f3 planar = rel_spin - normal * dot(rel_spin, normal);
    float planar_len = length(planar);
    if (planar_len > 1e-6f) {
        f3 axis = planar / planar_len;
        float mass = dot(axis, dbody_iinv(b.sf, axis)) + dot(axis, dbody_iinv(b.ss, axis));
        if (mass > 0.0f) {
            float limit = mat.x * normal_total;
            float applied = wclamp(-planar_len / mass, -limit, limit);
            first.angular_velocity = first.angular_velocity - dbody_iinv(first, axis * applied);
            second.angular_velocity = second.angular_velocity + dbody_iinv(second, axis * applied);
        }
    }
    float twist = dot(rel_spin, normal);
    if (fabsf(twist) > 1e-6f) {
        if (twist_mass > 0.0f) {
            float limit = mat.y * normal_total;
            float applied = wclamp(-twist / twist_mass, -limit, limit);
            first.angular_velocity = first.angular_velocity - dbody_iinv(first, normal * applied);
            second.angular_velocity = second.angular_velocity + dbody_iinv(second, normal * applied);
        }
    }
    f3 da = first.velocity - pf.velocity, sa = first.angular_velocity - pf.angular_velocity;
    f3 db = second.velocity - ps.velocity, sb = second.angular_velocity - ps.angular_velocity;
    if (!dbody_inert(pf)) accumulate(w.vdelta, r.x, da, sa, DYN_SOLVER_VELOCITY_SCALE);
    if (!dbody_inert(ps)) accumulate(w.vdelta, r.y, db, sb, DYN_SOLVER_VELOCITY_SCALE);
    if (residual) {
        max_counter(&w.counters[DYN_COUNTER_SOLVE_LINEAR_RESIDUAL],
                    (uint32_t)solver_word(wmax(length(da), length(db)), DYN_SOLVER_VELOCITY_SCALE));
        max_counter(&w.counters[DYN_COUNTER_SOLVE_ANGULAR_RESIDUAL],
                    (uint32_t)solver_word(wmax(length(sa), length(sb)), DYN_SOLVER_VELOCITY_SCALE));
    }
}
// tape_index: substep x iterations + iteration, where a taped step writes its snapshots
__global__ void __launch_bounds__(256, 2) k_solve(DeviceWorld w, dyn_step_params p, uint32_t tape_index) {
    const uint32_t count = w.ctl[CTL_CONTACTS];
    const bool residual = w.ctl[CTL_ROUNDS] == p.solve_iterations;
    GRID_STRIDE(i, count) solve_block(w, p, i, residual, tape_index);
}

// solver_block_apply.wgsl:7-29
__device__ __forceinline__ void apply_velocity_row(const DeviceWorld& w, uint32_t i) {
    uint32_t row = w.solver_rows[i];
    int4* d = reinterpret_cast<int4*>(w.vdelta + 8u * row);
    int4 a = d[0], b = d[1];
    d[0] = make_int4(0, 0, 0, 0);
    d[1] = make_int4(0, 0, 0, 0);
    f3 lin = mk3((float)a.x / DYN_SOLVER_VELOCITY_SCALE, (float)a.y / DYN_SOLVER_VELOCITY_SCALE,
                 (float)a.z / DYN_SOLVER_VELOCITY_SCALE);
    f3 ang = mk3((float)a.w / DYN_SOLVER_VELOCITY_SCALE, (float)b.x / DYN_SOLVER_VELOCITY_SCALE,
                 (float)b.y / DYN_SOLVER_VELOCITY_SCALE);
    if (is_zero3(lin) && is_zero3(ang)) return;
    BodyHot& h = w.hot[row];
    float4 v = h.vel, av = h.ang;
    h.vel = make_float4(v.x + lin.x, v.y + lin.y, v.z + lin.z, v.w);
    h.ang = make_float4(av.x + ang.x, av.y + ang.y, av.z + ang.z, av.w);
}
__global__ void k_vapply(DeviceWorld w) {
    const uint32_t rows = w.ctl[CTL_SOLVER_ROWS];
    if (blockIdx.x == 0 && threadIdx.x == 0 && rows > 0u) w.ctl[CTL_ROUNDS] += 1u;
    GRID_STRIDE(i, rows) apply_velocity_row(w, i);
}

// substep_integrate.wgsl:15-76 (no force fields)
__global__ void k_integrate(DeviceWorld w, dyn_step_params p) {
    const uint32_t live = w.ctl[CTL_LIVE];
    if (blockIdx.x == 0 && threadIdx.x == 0 && live > 0u) w.ctl[CTL_ROUNDS] = 0u;
    const float h = p.substep_dt;
    GRID_STRIDE(i, live) {
        uint32_t row = w.live[i];
        BodyHot& b = w.hot[row];
        float im = b.pos.w;
        uint32_t flags = b.aux.y;
        if (!simulates(im, flags)) continue;
        float4 q = b.rot;
        float4 dm = w.damp[row];
        f3 force = xyz(w.force[row]), torque = xyz(w.torque[row]);
        f3 acceleration = mk3(p.gravity[0], p.gravity[1], p.gravity[2]) * dm.z + force * im;
        f3 spin = xyz(b.ang);
        f3 velocity = xyz(b.vel) + acceleration * h;
        float4 ii0 = b.ii0;
        float2 ii1 = make_float2(b.ii1.x, b.ii1.y);
        float4 I0 = w.inert0[row];
        float2 I1 = w.inert1[row];
        f3 gyro = spin;
        bool isotropic = I0.y == 0.0f && I0.z == 0.0f && I1.x == 0.0f && I0.x == I0.w && I0.w == I1.y;
        if (!isotropic) {
            f3 body_spin = quat_rotate(quat_conj(q), spin);
            f3 momentum = sym_apply(I0, I1, body_spin);
            if (!is_zero3(cross(body_spin, momentum))) {
                f3 solved = momentum;
                for (int it = 0; it < 4; ++it) {
                    f3 mid = 0.5f * (momentum + solved);
                    solved = rotate_about(-sym_apply(ii0, ii1, mid) * h, momentum);
                }
                gyro = quat_rotate(q, sym_apply(ii0, ii1, solved));
            }
        }
        f3 angular = gyro + inv_inertia_world(ii0, ii1, q, torque * h);
        float speed = length(velocity);
        if (speed > p.max_velocity) velocity = velocity * (p.max_velocity / speed);
        float spin_speed = length(angular);
        if (spin_speed > p.max_angular_velocity) angular = angular * (p.max_angular_velocity / spin_speed);
        velocity = velocity / (1.0f + dm.x * h);
        angular = angular / (1.0f + dm.y * h);
        b.vel = mk4(velocity, 0.0f);
        b.ang = mk4(angular, 0.0f);
    }
}

// substep_advance.wgsl:6-13
__global__ void k_advance(DeviceWorld w, dyn_step_params p) {
    const uint32_t live = w.ctl[CTL_LIVE];
    const float h = p.substep_dt;
    GRID_STRIDE(i, live) {
        uint32_t row = w.live[i];
        BodyHot& b = w.hot[row];
        f3 pos = xyz(b.pos) + xyz(b.vel) * h;
        float4 q = b.rot;
        f3 av = xyz(b.ang);
        float4 spin = make_float4(av.x, av.y, av.z, 0.0f);
        b.pos = mk4(pos, b.pos.w);
        b.rot = normalize4(add4(q, scale4(0.5f * h, quat_mul(spin, q))));
    }
}

// position_correction.wgsl:5-46 with position_block.wgsl:11-33
__device__ __forceinline__ void position_block(const DeviceWorld& w, const dyn_step_params& p, uint32_t i) {
    const uint32_t cap = w.c_cap;
    uint4 r = w.cur.rows[i];
    if (!resolves(r)) return;
    float4 mat = w.cur.mat[i];
    if (mat.z > 0.0f) return;
    const BodyHot& ha = w.hot[r.x];
    const BodyHot& hb = w.hot[r.y];
    float ima = (!simulates(ha.pos.w, ha.aux.y) || ha.aux.x != 0u) ? 0.0f : ha.pos.w;
    float imb = (!simulates(hb.pos.w, hb.aux.y) || hb.aux.x != 0u) ? 0.0f : hb.pos.w;
    f3 normal = xyz(w.cur.normal[i]);
    float resolved = dot(normal, xyz(w.resolution[r.y]) - xyz(w.resolution[r.x]));
    f3 total = s3(0.0f);
    uint32_t contributing = 0;
    uint32_t pc = r.z & 0xFFu;
    for (uint32_t pi = 0; pi < pc; ++pi) {
        float error = wmax(w.cur.la[(size_t)pi * cap + i].w - p.slop - resolved, 0.0f);
        if (error <= 0.0f) continue;
        float k = ima + imb;
        if (k == 0.0f) continue;
        total = total + normal * (p.relaxation * error / k);
        contributing += 1;
    }
    if (contributing == 0u) return;
    f3 correction = total / (float)contributing;
    f3 la = -correction * ima;
    f3 lb = correction * imb;
    if (!(dot(la, la) > 0.0f || dot(lb, lb) > 0.0f)) return;
    // Both rows are marked as contributing (position_apply renormalises a contributed row's
    // orientation). A moving row needs the exact count, which divides its summed delta; a
    // frozen row's sum is zero, so only "contributed" matters there: every writer stores the
    // same 1, without an atomic on the shared row of a static body.
    if (ima > 0.0f) {
        atomicAdd(&w.contributions[r.x], 1u);
        accumulate_linear(w.pdelta, r.x, la, DYN_SOLVER_POSITION_SCALE);
    } else if (w.contributions[r.x] == 0u) {
        w.contributions[r.x] = 1u;
    }
    if (imb > 0.0f) {
        atomicAdd(&w.contributions[r.y], 1u);
        accumulate_linear(w.pdelta, r.y, lb, DYN_SOLVER_POSITION_SCALE);
    } else if (w.contributions[r.y] == 0u) {
        w.contributions[r.y] = 1u;
    }
}
__global__ void k_position(DeviceWorld w, dyn_step_params p) {
    const uint32_t count = w.ctl[CTL_CONTACTS];
    GRID_STRIDE(i, count) position_block(w, p, i);
}

// position_apply.wgsl:12-27
__device__ __forceinline__ void apply_position_row(const DeviceWorld& w, uint32_t i) {
    uint32_t row = w.solver_rows[i];
    uint32_t contributing = w.contributions[row];
    w.contributions[row] = 0u;
    int4* d = reinterpret_cast<int4*>(w.pdelta + 8u * row);
    int4 a = d[0], b = d[1];
    d[0] = make_int4(0, 0, 0, 0);
    d[1] = make_int4(0, 0, 0, 0);
    if (contributing == 0u) return;
    f3 lin = mk3((float)a.x / DYN_SOLVER_POSITION_SCALE, (float)a.y / DYN_SOLVER_POSITION_SCALE,
                 (float)a.z / DYN_SOLVER_POSITION_SCALE);
    f3 ang = mk3((float)a.w / DYN_SOLVER_POSITION_SCALE, (float)b.x / DYN_SOLVER_POSITION_SCALE,
                 (float)b.y / DYN_SOLVER_POSITION_SCALE);
    f3 al = lin / (float)contributing;
    f3 aa = ang / (float)contributing;
    BodyHot& h = w.hot[row];
    f3 pos = xyz(h.pos) + al;
    h.pos = mk4(pos, h.pos.w);
    f3 ha = aa * 0.5f;
    h.rot = normalize4(quat_mul(make_float4(ha.x, ha.y, ha.z, 1.0f), h.rot));
    float4 res = w.resolution[row];
    w.resolution[row] = make_float4(res.x + al.x, res.y + al.y, res.z + al.z, 0.0f);
}
__global__ void k_papply(DeviceWorld w) {
    const uint32_t rows = w.ctl[CTL_SOLVER_ROWS];
    GRID_STRIDE(i, rows) apply_position_row(w, i);
}

// ---- the position pass with its apply folded into the next iteration (worlds without joints) ----
// Iteration k of a substep's position loop needs each row's resolution after iteration k-1's
// correction: the row's summed delta over its contribution count, as position_apply.wgsl:12-27
// forms it. Every contact forms it where it reads it, from iteration k-1's delta words; the row's
// owner (the contact that claimed the row in k_solver_blocks) also stores it and moves the row's
// pose. Three delta buffers rotate: k-1's are read, k's are summed into, k+1's are cleared by the
// owners (nothing reads or writes them during iteration k). The integers and the float operations
// are k_papply's, so poses and resolutions come out bit for bit as with the separate apply, one
// launch per iteration fewer; k_papply_last applies the last iteration. Joint passes move bodies
// between the contact iterations, so worlds with joints keep the separate apply.
struct RowCorrection {
    f3 al;
    uint32_t contributing;
};
__device__ __forceinline__ RowCorrection row_correction(const int4* __restrict__ pd, const uint32_t* __restrict__ cnt, uint32_t row) {
    RowCorrection c;
    c.contributing = cnt[row];
    c.al = s3(0.0f);
    if (c.contributing != 0u) {
        const int4 a = pd[row];
        const f3 lin = mk3((float)a.x / DYN_SOLVER_POSITION_SCALE, (float)a.y / DYN_SOLVER_POSITION_SCALE,
                           (float)a.z / DYN_SOLVER_POSITION_SCALE);
        c.al = lin / (float)c.contributing;
    }
    return c;
}
__device__ __forceinline__ float4 corrected(float4 res, const RowCorrection& c) {
    if (c.contributing == 0u) return res;
    return make_float4(res.x + c.al.x, res.y + c.al.y, res.z + c.al.z, 0.0f);
}
// apply_position_row's pose update: a pure translation, and the orientation renormalised
__device__ __forceinline__ void move_row(const DeviceWorld& w, uint32_t row, const RowCorrection& c) {
    if (c.contributing == 0u) return;
    const f3 aa = s3(0.0f) / (float)c.contributing;
    BodyHot& h = w.hot[row];
    const f3 pos = xyz(h.pos) + c.al;
    h.pos = mk4(pos, h.pos.w);
    const f3 ha = aa * 0.5f;
    h.rot = normalize4(quat_mul(make_float4(ha.x, ha.y, ha.z, 1.0f), h.rot));
}
__device__ __forceinline__ void position_block_rows(const DeviceWorld& w, const dyn_step_params& p, uint32_t i, uint4 r,
                                                    float4 res_a, float4 res_b, int4* __restrict__ pd,
                                                    uint32_t* __restrict__ cnt) {
    const uint32_t cap = w.c_cap;
    if (!resolves(r)) return;
    float4 mat = w.cur.mat[i];
    if (mat.z > 0.0f) return;
    const BodyHot& ha = w.hot[r.x];
    const BodyHot& hb = w.hot[r.y];
    float ima = (!simulates(ha.pos.w, ha.aux.y) || ha.aux.x != 0u) ? 0.0f : ha.pos.w;
    float imb = (!simulates(hb.pos.w, hb.aux.y) || hb.aux.x != 0u) ? 0.0f : hb.pos.w;
    f3 normal = xyz(w.cur.normal[i]);
    float resolved = dot(normal, xyz(res_b) - xyz(res_a));
    f3 total = s3(0.0f);
    uint32_t contributing = 0;
    uint32_t pc = r.z & 0xFFu;
    for (uint32_t pi = 0; pi < pc; ++pi) {
        float error = wmax(w.cur.la[(size_t)pi * cap + i].w - p.slop - resolved, 0.0f);
        if (error <= 0.0f) continue;
        float k = ima + imb;
        if (k == 0.0f) continue;
        total = total + normal * (p.relaxation * error / k);
        contributing += 1;
    }
    if (contributing == 0u) return;
    f3 correction = total / (float)contributing;
    f3 la = -correction * ima;
    f3 lb = correction * imb;
    if (!(dot(la, la) > 0.0f || dot(lb, lb) > 0.0f)) return;
    int32_t* da = reinterpret_cast<int32_t*>(pd + r.x);
    int32_t* db = reinterpret_cast<int32_t*>(pd + r.y);
    if (ima > 0.0f) {
        atomicAdd(&cnt[r.x], 1u);
        atomicAdd(da + 0, solver_word(la.x, DYN_SOLVER_POSITION_SCALE));
        atomicAdd(da + 1, solver_word(la.y, DYN_SOLVER_POSITION_SCALE));
        atomicAdd(da + 2, solver_word(la.z, DYN_SOLVER_POSITION_SCALE));
    } else if (cnt[r.x] == 0u) {
        cnt[r.x] = 1u;
    }
    if (imb > 0.0f) {
        atomicAdd(&cnt[r.y], 1u);
        atomicAdd(db + 0, solver_word(lb.x, DYN_SOLVER_POSITION_SCALE));
        atomicAdd(db + 1, solver_word(lb.y, DYN_SOLVER_POSITION_SCALE));
        atomicAdd(db + 2, solver_word(lb.z, DYN_SOLVER_POSITION_SCALE));
    } else if (cnt[r.y] == 0u) {
        cnt[r.y] = 1u;
    }
}
// A taped step's position snapshots, written by each solver row's owner: the resolution iteration
// k starts from, and the contributions iteration k - 1 counted.
__device__ __forceinline__ void tape_position_row(const TapeWrites& t, uint32_t sub, uint32_t k, uint32_t row, float4 res,
                                                  bool with_count, uint32_t count) {
    const size_t slot = *t.slot;
    const size_t base = slot * t.substeps * t.piterations + (size_t)sub * t.piterations;
    t.res[(base + k) * t.n + row] = res;
    if (with_count) t.cnt[(base + k - 1u) * t.n + row] = count;
}
template <bool kFirst>
__global__ void k_position_fused(DeviceWorld w, dyn_step_params p, uint32_t k, uint32_t sub) {
    const uint32_t count = w.ctl[CTL_CONTACTS];
    const size_t n = w.n_cap;
    const int4* pd_prev = w.pd3 + ((k + 2u) % 3u) * n;
    int4* pd_cur = w.pd3 + (k % 3u) * n;
    int4* pd_next = w.pd3 + ((k + 1u) % 3u) * n;
    const uint32_t* cnt_prev = w.cnt3 + ((k + 2u) % 3u) * n;
    uint32_t* cnt_cur = w.cnt3 + (k % 3u) * n;
    uint32_t* cnt_next = w.cnt3 + ((k + 1u) % 3u) * n;
    const float4* res_prev = ((k + 1u) & 1u) ? w.resolution_alt : w.resolution;
    float4* res_cur = (k & 1u) ? w.resolution_alt : w.resolution;
    GRID_STRIDE(i, count) {
        const uint4 r = w.cur.rows[i];
        float4 res_a, res_b;
        if (kFirst) {
            res_a = w.resolution[r.x];
            res_b = w.resolution[r.y];
            if (w.tape.res) {
                const uint32_t own = w.cowner[i];
                if (own & 1u) tape_position_row(w.tape, sub, 0u, r.x, res_a, false, 0u);
                if (own & 2u) tape_position_row(w.tape, sub, 0u, r.y, res_b, false, 0u);
            }
        } else {
            const RowCorrection ca = row_correction(pd_prev, cnt_prev, r.x);
            const RowCorrection cb = row_correction(pd_prev, cnt_prev, r.y);
            res_a = corrected(res_prev[r.x], ca);
            res_b = corrected(res_prev[r.y], cb);
            const uint32_t own = w.cowner[i];
            if (w.tape.res) {
                if (own & 1u) tape_position_row(w.tape, sub, k, r.x, res_a, true, ca.contributing);
                if (own & 2u) tape_position_row(w.tape, sub, k, r.y, res_b, true, cb.contributing);
            }
            if (own & 1u) {
                res_cur[r.x] = res_a;
                move_row(w, r.x, ca);
                pd_next[r.x] = make_int4(0, 0, 0, 0);
                cnt_next[r.x] = 0u;
            }
            if (own & 2u) {
                res_cur[r.y] = res_b;
                move_row(w, r.y, cb);
                pd_next[r.y] = make_int4(0, 0, 0, 0);
                cnt_next[r.y] = 0u;
            }
        }
        position_block_rows(w, p, i, r, res_a, res_b, pd_cur, cnt_cur);
    }
}
// The last iteration's correction of every solver row, into the resolution every later pass reads;
// the three delta buffers are left cleared for the next substep.
__global__ void k_papply_last(DeviceWorld w, uint32_t iterations, uint32_t sub) {
    const uint32_t rows = w.ctl[CTL_SOLVER_ROWS];
    const size_t n = w.n_cap;
    const uint32_t last = iterations - 1u;
    const int4* pd_last = w.pd3 + (last % 3u) * n;
    const uint32_t* cnt_last = w.cnt3 + (last % 3u) * n;
    const float4* res_last = (last & 1u) ? w.resolution_alt : w.resolution;
    GRID_STRIDE(i, rows) {
        const uint32_t row = w.solver_rows[i];
        const RowCorrection c = row_correction(pd_last, cnt_last, row);
        if (w.tape.cnt) {  // a taped step: the last iteration's contributions
            const size_t slot = *w.tape.slot;
            w.tape.cnt[(slot * w.tape.substeps * w.tape.piterations + (size_t)sub * w.tape.piterations + last) * w.tape.n + row] =
                c.contributing;
        }
        const float4 res = corrected(res_last[row], c);
        w.resolution[row] = res;
        move_row(w, row, c);
        for (uint32_t b = 0; b < 3u; ++b) {
            w.pd3[b * n + row] = make_int4(0, 0, 0, 0);
            w.cnt3[b * n + row] = 0u;
        }
    }
}

// island_sleep.wgsl:10-29, then commit (contact_archive + archive_count_sync).
__global__ void k_sleep(DeviceWorld w, dyn_step_params p) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        w.ctl[CTL_ARCHIVED] = w.ctl[CTL_CONTACTS];
        w.counters[DYN_COUNTER_ARCHIVED] = w.ctl[CTL_CONTACTS];
        w.counters[DYN_COUNTER_LIVE] = w.ctl[CTL_LIVE];
        w.counters[DYN_COUNTER_SOLVER_ROWS] = w.ctl[CTL_SOLVER_ROWS];
        w.counters[DYN_COUNTER_STEP] += 1u;
        // the host reads the pair demand (the largest since it last looked) and any refusal, and
        // widens the pair stream before a later step
        if (w.spill != nullptr) {
            const uint32_t refused = w.counters[DYN_COUNTER_REFUSED_PAIRS];
            const uint32_t demand = w.counters[DYN_COUNTER_PAIRS];
            if (demand > w.spill[1]) w.spill[1] = demand;
            if (refused != 0u) w.spill[2] = refused;
            const uint32_t contacts = w.ctl[CTL_STAGED];
            if (contacts > w.spill[3]) w.spill[3] = contacts;
        }
    }
    GRID_STRIDE(i, w.nd) {
        BodyHot& h = w.hot[i];
        if (h.aux.x != 0u || !simulates(h.pos.w, h.aux.y)) continue;
        uint32_t root = w.parents[i];
        bool disturbed = (w.istate[root] & DYN_ISLAND_WAKE) != 0u || w.wake_flags[i] != 0u;
        if (disturbed) {
            w.sleep_timer[i] = 0.0f;
        } else {
            float t = w.sleep_timer[i] + p.dt;
            if (t >= p.sleep_time) {
                h.vel = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                h.ang = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                w.force[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                w.torque[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                w.prev_pos[i] = make_float4(h.pos.x, h.pos.y, h.pos.z, 0.0f);
                w.prev_rot[i] = h.rot;
                t = 0.0f;
                h.aux.x = 1u;
                add_counter(&w.counters[DYN_COUNTER_SLEPT], 1u);
            }
            w.sleep_timer[i] = t;
        }
    }
}

// ---- ABI state records <-> device layout (one contiguous copy each way) ----
__global__ void k_unpack_states(DeviceWorld w, const dyn_body_state_record* __restrict__ in, uint32_t n) {
    GRID_STRIDE(i, n) {
        const dyn_body_state_record& r = in[i];
        BodyHot& h = w.hot[i];
        h.pos = make_float4(r.position[0], r.position[1], r.position[2], h.pos.w);
        h.rot = make_float4(r.orientation[0], r.orientation[1], r.orientation[2], r.orientation[3]);
        h.vel = make_float4(r.velocity[0], r.velocity[1], r.velocity[2], 0.0f);
        h.ang = make_float4(r.angular_velocity[0], r.angular_velocity[1], r.angular_velocity[2], 0.0f);
        h.aux.x = r.sleeping;
        w.prev_pos[i] = make_float4(r.prev_position[0], r.prev_position[1], r.prev_position[2], 0.0f);
        w.prev_rot[i] = make_float4(r.prev_orientation[0], r.prev_orientation[1], r.prev_orientation[2], r.prev_orientation[3]);
        w.force[i] = make_float4(r.force[0], r.force[1], r.force[2], 0.0f);
        w.torque[i] = make_float4(r.torque[0], r.torque[1], r.torque[2], 0.0f);
        w.sleep_timer[i] = r.sleep_timer;
    }
}
__device__ __forceinline__ void pack_state(const DeviceWorld& w, uint32_t i, dyn_body_state_record* __restrict__ dst) {
    const BodyHot& h = w.hot[i];
    float4 pp = w.prev_pos[i], pr = w.prev_rot[i], f = w.force[i], t = w.torque[i];
    uint4 id = w.ident[i];
    dyn_body_state_record r;
    r.position[0] = h.pos.x; r.position[1] = h.pos.y; r.position[2] = h.pos.z; r._pad0 = 0.0f;
    r.prev_position[0] = pp.x; r.prev_position[1] = pp.y; r.prev_position[2] = pp.z; r._pad1 = 0.0f;
    r.prev_orientation[0] = pr.x; r.prev_orientation[1] = pr.y; r.prev_orientation[2] = pr.z; r.prev_orientation[3] = pr.w;
    r.orientation[0] = h.rot.x; r.orientation[1] = h.rot.y; r.orientation[2] = h.rot.z; r.orientation[3] = h.rot.w;
    r.velocity[0] = h.vel.x; r.velocity[1] = h.vel.y; r.velocity[2] = h.vel.z; r._pad2 = 0.0f;
    r.angular_velocity[0] = h.ang.x; r.angular_velocity[1] = h.ang.y; r.angular_velocity[2] = h.ang.z; r._pad3 = 0.0f;
    r.force[0] = f.x; r.force[1] = f.y; r.force[2] = f.z; r._pad4 = 0.0f;
    r.torque[0] = t.x; r.torque[1] = t.y; r.torque[2] = t.z; r._pad5 = 0.0f;
    r.body_id = id.x;
    r.generation = id.y;
    r.sleep_timer = w.sleep_timer[i];
    r.sleeping = h.aux.x;
    *dst = r;
}
__global__ void k_pack_states(DeviceWorld w, dyn_body_state_record* __restrict__ out, uint32_t n) {
    GRID_STRIDE(i, n) pack_state(w, i, out + i);
}
// The state records of the listed bodies, in list order (the observation ring's copies); a body
// that is not in the world gets a record with body_id DYN_NO_BODY.
__global__ void k_pack_ids(DeviceWorld w, const uint32_t* __restrict__ ids, dyn_body_state_record* __restrict__ out,
                           uint32_t m) {
    GRID_STRIDE(i, m) {
        const uint32_t id = ids[i];
        const uint32_t row = id < w.id_count ? w.row_of_id[id] : DYN_NO_BODY;
        if (row < w.n) {
            pack_state(w, row, out + i);
        } else {
            out[i].body_id = DYN_NO_BODY;
        }
    }
}

}  // namespace dyn
