// ccd.cuh - continuous collision: every candidate pair with a body that declares CCD is swept over
// the step's motion, and each such body retreats to its earliest impact
// (crates/dynamis-rigid/src/ccd.rs:1-113; shaders/ccd_sweep.wgsl:1-211, shaders/ccd_apply.wgsl:1-38).
// The passes run after the substeps and before sleep, and only in worlds that hold a CCD body (the
// reference's CCD_GATE, crates/dynamis-rigid/src/domain.rs:85-96).
//
// The reference publishes an impact with an atomicMin on the time and a plain store of the impact
// record by whichever invocation lowered it (ccd_sweep.wgsl:158-168), so at equal times the record
// kept depends on invocation order. Here the choice is fixed: the earliest time, then the lowest
// (lower, higher collider slot) pair key. Four kernels:
//   k_ccd_sweep  (pair)  sweeps both directions of a pair, records each hit in a list, and keeps the
//                        earliest time per body (atomicMax on the complement of the time bits: the
//                        times are non-negative floats, whose bit patterns order like the values);
//   k_ccd_pick   (hit)   among a body's earliest hits, keeps the lowest pair key;
//   k_ccd_impact (hit)   the hit holding both writes the body's impact record;
//   k_ccd_apply  (row)   ccd_apply.wgsl, then clears the row's words for the next step.
// The hit list reuses the separated-pair probe queue of the narrowphase (probe_data, six float4 per
// pair slot), which nothing reads after the narrowphase: a pair yields at most two hits, three
// float4 each.
#pragma once

#include "narrow.cuh"
#include "step.cuh"

namespace dyn {

constexpr uint32_t kSweepIterations = 16u;  // ccd_sweep.wgsl:15
constexpr float kSweepTolerance = 1e-4f;    // SWEEP_TOLERANCE, crates/dynamis-shader/shaders/scene.wgsl:1
constexpr float kNoHit = 3.402823466e38f;   // NO_HIT

// core.wgsl:149-163
__device__ __forceinline__ float4 quat_slerp(float4 a, float4 b, float t) {
    float cosine = dot4(a, b);
    if (cosine < 0.0f) {
        b = make_float4(-b.x, -b.y, -b.z, -b.w);
        cosine = -cosine;
    }
    if (cosine > 0.9995f) {
        return normalize4(make_float4(a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t, a.z + (b.z - a.z) * t,
                                      a.w + (b.w - a.w) * t));
    }
    const float angle = dacos(wclamp(cosine, -1.0f, 1.0f));
    const float sine = dsin(angle);
    const float wa = dsin((1.0f - t) * angle) / sine, wb = dsin(t * angle) / sine;
    return make_float4(a.x * wa + b.x * wb, a.y * wa + b.y * wb, a.z * wa + b.z * wb, a.w * wa + b.w * wb);
}
// core.wgsl:165-168
__device__ __forceinline__ float quat_angle(float4 a, float4 b) {
    return 2.0f * dacos(fabsf(wclamp(dot4(a, b), -1.0f, 1.0f)));
}

// A body's pose at fraction t of the step's motion (ccd_sweep.wgsl:40-45).
struct SweptBody {
    DBody body;
    f3 prev_position;
    float4 prev_orientation;
};
__device__ __forceinline__ SweptBody load_swept(const DeviceWorld& w, uint32_t row) {
    SweptBody s;
    s.body = load_dbody(w.hot, row);
    s.prev_position = xyz(w.prev_pos[row]);
    s.prev_orientation = w.prev_rot[row];
    return s;
}
__device__ __forceinline__ WShape swept_shape(const SweptBody& s, const DColl& c, float t) {
    const f3 position = s.prev_position + (s.body.position - s.prev_position) * t;
    return world_shape(position, quat_slerp(s.prev_orientation, s.body.orientation, t), c);
}

struct SweepReach {
    float travel, spin;
};
// ccd_sweep.wgsl:47-61
__device__ __forceinline__ float sweep_radius(const DeviceWorld& w, const DBody& b, const DColl& c) {
    if (c.kind == DYN_SHAPE_PLANE) return 0.0f;
    const DAabb bounds = world_aabb(w, world_shape(b.position, b.orientation, c));
    const f3 center = b.position + quat_rotate(b.orientation, c.offset);
    return length((bounds.max - bounds.min) * 0.5f) + length(center - dbody_com(b));
}
__device__ __forceinline__ SweepReach sweep_reach(const DeviceWorld& w, const SweptBody& s, const DColl& c) {
    SweepReach r;
    r.travel = length(s.body.position - s.prev_position);
    r.spin = quat_angle(s.prev_orientation, s.body.orientation) * sweep_radius(w, s.body, c);
    return r;
}

// ccd_sweep.wgsl:63-69
__device__ __forceinline__ Hit plane_convex_gap(const DeviceWorld& w, const WShape& plane, const WShape& convex) {
    const f3 normal = quat_rotate(plane.rotation, mk3(0.0f, 1.0f, 0.0f));
    const float side = dot(convex.center - plane.center, normal);
    const f3 facing = side < 0.0f ? -normal : normal;
    const float extent = dot(support(w, convex, facing) - convex.center, facing);
    return Hit{fabsf(side) - extent, convex.center + facing * extent, facing};
}
// ccd_sweep.wgsl:71-98. Triangle scenes (meshes, heightfields) are refused when a scene is built, so
// their branch answers no hit.
__device__ __forceinline__ Hit pair_gap(const DeviceWorld& w, const WShape& first, const WShape& second) {
    if (first.kind == DYN_SHAPE_PLANE) {
        const Hit swapped = plane_convex_gap(w, first, second);
        return Hit{swapped.distance, swapped.point, -swapped.normal};
    }
    if (second.kind == DYN_SHAPE_PLANE) return plane_convex_gap(w, second, first);
    if (shape_world_geometry(first.kind) || shape_world_geometry(second.kind)) return Hit{kNoHit, s3(0.0f), s3(0.0f)};
    return convex_hit(w, first, second);
}

struct SweepHit {
    float time;
    f3 normal, point;
};
// ccd_sweep.wgsl:100-147
__device__ SweepHit rigid_sweep(const DeviceWorld& w, const SweptBody& moving, const DColl& mc, const SweptBody& other,
                                const DColl& oc) {
    SweepHit none{1.0f, mk3(0.0f, 1.0f, 0.0f), s3(0.0f)};
    if ((moving.body.flags & DYN_BODY_CCD) == 0u) return none;
    const SweepReach free_reach = sweep_reach(w, moving, mc);
    const bool other_movable = moves(other.body.inverse_mass, other.body.flags);
    SweepReach other_reach{0.0f, 0.0f};
    if (other_movable) other_reach = sweep_reach(w, other, oc);
    const float closing_floor = free_reach.spin + other_reach.spin;
    if (free_reach.travel + closing_floor + other_reach.travel <= 0.0f) return none;
    const f3 free_travel = moving.body.position - moving.prev_position;
    const f3 other_travel = other_movable ? other.body.position - other.prev_position : s3(0.0f);
    float t = 0.0f;
    for (uint32_t iteration = 0; iteration < kSweepIterations; ++iteration) {
        const WShape free = swept_shape(moving, mc, t);
        const WShape fixed = other_movable ? swept_shape(other, oc, t)
                                           : world_shape(other.body.position, other.body.orientation, oc);
        const Hit gap = pair_gap(w, free, fixed);
        if (gap.distance <= kSweepTolerance) {
            if (iteration == 0u && gap.distance <= 0.0f) return none;
            const f3 point = free.kind == DYN_SHAPE_PLANE ? free.center : support(w, free, gap.normal);
            return SweepHit{t, gap.normal, point};
        }
        const float closing = dot(free_travel - other_travel, gap.normal) + closing_floor;
        if (closing <= 0.0f) return none;
        t = t + gap.distance / closing;
        if (t >= 1.0f) return none;
    }
    return none;
}

// One direction of a pair: the moving body's hit, if any, into the hit list (ccd_sweep.wgsl:149-186).
__device__ __forceinline__ void retreat(const DeviceWorld& w, const dyn_step_params& p, uint32_t row, const SweptBody& moving,
                                        const DColl& mc, uint32_t mslot, const SweptBody& other, const DColl& oc,
                                        uint32_t oslot, uint32_t major, uint32_t minor) {
    const SweepHit hit = rigid_sweep(w, moving, mc, other, oc);
    if (!(hit.time < 1.0f)) return;
    const float a = w.c_mat[mslot].y, b = w.c_mat[oslot].y;
    const uint32_t mode = p.restitution_combine;
    const float restitution = mode == 1u ? wmin(a, b) : (mode == 2u ? wmax(a, b) : (mode == 3u ? (a + b) * 0.5f : sqrtf(a * b)));
    const uint32_t slot = append_slot(&w.ctl[CTL_CCD_HITS]);
    if (slot >= 2u * w.p_cap) return;  // a pair records at most two hits: unreachable
    w.probe_data[3 * (size_t)slot] = mk4(sign_normalize(hit.normal), restitution);
    w.probe_data[3 * (size_t)slot + 1] = mk4(hit.point, hit.time);
    w.probe_data[3 * (size_t)slot + 2] = make_float4(__uint_as_float(row), __uint_as_float(major), __uint_as_float(minor), 0.0f);
    atomicMax(&w.ccd_time[row], ~__float_as_uint(hit.time));
}

// ccd_sweep.wgsl:188-211 (the pairs are unique, so the sorted list's duplicate check has nothing to skip)
__global__ void __launch_bounds__(128) k_ccd_sweep(DeviceWorld w, dyn_step_params p) {
    const uint32_t pairs = min(w.counters[DYN_COUNTER_PAIRS], w.p_cap);
    GRID_STRIDE(index, pairs) {
        const uint32_t fs = w.pmaj[index], ss = w.pmin[index];
        const uint4 f = w.c_class[fs], s = w.c_class[ss];
        const uint32_t fr = f.x, sr = s.x;
        if (fr == DYN_NO_BODY || sr == DYN_NO_BODY || fr == sr) continue;
        // only a body that declares CCD sweeps (rigid_sweep's first test), so the other pairs stop here
        if (((w.hot[fr].aux.y | w.hot[sr].aux.y) & DYN_BODY_CCD) == 0u) continue;
        if (((f.w | s.w) & 0x100u) == 0u) continue;                   // neither body moves
        if ((f.w & 0xffu) == 0u || (s.w & 0xffu) == 0u) continue;     // SHAPE_NONE
        if (!((f.y & s.z) != 0u && (s.y & f.z) != 0u)) continue;      // collision filters
        if (joined_by_joint(w, fr, sr)) continue;
        const SweptBody first = load_swept(w, fr), second = load_swept(w, sr);
        const DColl fc = load_dcoll(w, fs), sc = load_dcoll(w, ss);
        retreat(w, p, fr, first, fc, fs, second, sc, ss, fs, ss);
        retreat(w, p, sr, second, sc, ss, first, fc, fs, fs, ss);
    }
}

__device__ __forceinline__ unsigned long long ccd_pair_key(uint32_t major, uint32_t minor) {
    return ((unsigned long long)major << 32) | minor;
}

// Among each body's hits at its earliest time, the lowest pair key.
__global__ void k_ccd_pick(DeviceWorld w) {
    const uint32_t hits = min(w.ctl[CTL_CCD_HITS], 2u * w.p_cap);
    GRID_STRIDE(h, hits) {
        const float4 at = w.probe_data[3 * (size_t)h + 1], meta = w.probe_data[3 * (size_t)h + 2];
        const uint32_t row = __float_as_uint(meta.x);
        if (~__float_as_uint(at.w) != w.ccd_time[row]) continue;
        atomicMax(&w.ccd_key[row], ~ccd_pair_key(__float_as_uint(meta.y), __float_as_uint(meta.z)));
    }
}

// The hit holding both the earliest time and the lowest key writes the body's impact.
__global__ void k_ccd_impact(DeviceWorld w) {
    const uint32_t hits = min(w.ctl[CTL_CCD_HITS], 2u * w.p_cap);
    GRID_STRIDE(h, hits) {
        const float4 at = w.probe_data[3 * (size_t)h + 1], meta = w.probe_data[3 * (size_t)h + 2];
        const uint32_t row = __float_as_uint(meta.x);
        if (~__float_as_uint(at.w) != w.ccd_time[row]) continue;
        if (~ccd_pair_key(__float_as_uint(meta.y), __float_as_uint(meta.z)) != w.ccd_key[row]) continue;
        w.ccd_impact[2 * (size_t)row] = w.probe_data[3 * (size_t)h];
        w.ccd_impact[2 * (size_t)row + 1] = at;
    }
}

// ccd_apply.wgsl:7-37 over the dynamic rows; every row's words are cleared for the next step (a
// body without a hit has none to clear, the reference's begin_step.wgsl:6 resets the factor).
__global__ void k_ccd_apply(DeviceWorld w) {
    GRID_STRIDE(row, w.n) {
        const uint32_t word = w.ccd_time[row];
        if (word == 0u) continue;
        w.ccd_time[row] = 0u;
        w.ccd_key[row] = 0ull;
        if (row >= w.nd) continue;
        const float time = __uint_as_float(~word);
        const float4 n4 = w.ccd_impact[2 * (size_t)row], p4 = w.ccd_impact[2 * (size_t)row + 1];
        const f3 axis = xyz(n4);
        const float restitution = n4.w;
        BodyHot& h = w.hot[row];
        DBody b = load_dbody(w.hot, row);
        const f3 lever = xyz(p4) - dbody_com(b);
        const f3 arm = cross(lever, axis);
        const float linear_speed = dot(b.velocity, axis);
        const float angular_speed = dot(b.angular_velocity, arm);
        if (linear_speed <= 0.0f && angular_speed <= 0.0f) continue;
        const f3 prev_position = xyz(w.prev_pos[row]);
        b.position = prev_position + (b.position - prev_position) * time;
        b.orientation = quat_slerp(w.prev_rot[row], b.orientation, time);
        if (linear_speed > 0.0f) b.velocity = b.velocity - axis * (linear_speed * (1.0f + restitution));
        if (angular_speed > 0.0f) {
            const float mass = b.inverse_mass + dot(arm, dbody_iinv(b, arm));
            if (mass > 0.0f) {
                const float impulse = angular_speed * (1.0f + restitution) / mass;
                b.velocity = b.velocity - axis * (impulse * b.inverse_mass);
                b.angular_velocity = b.angular_velocity - dbody_iinv(b, arm * impulse);
            }
        }
        h.pos = mk4(b.position, b.inverse_mass);
        h.rot = b.orientation;
        h.vel = mk4(b.velocity, 0.0f);
        h.ang = mk4(b.angular_velocity, 0.0f);
    }
}

}  // namespace dyn
