// query.cuh - scene queries over the grid: rays, sphere / point / cuboid / convex overlaps and
// convex sweeps against the colliders (crates/dynamis-shader/shaders/scene_cast.wgsl:1-534 for the
// candidate walk and the hit selection; scene.wgsl:1-258, 259-320, 813-873 for the hit tests).
//
// One block per query. The candidates are the colliders with an entry in the grid cells the
// query's box covers, level by level (grid_index.wgsl:289-388: a level whose cells under the box
// number more than GRID_WALK_CELLS is scanned whole, entries tested against the box; otherwise its
// cells are looked up one by one), at most QUERY_CANDIDATES of them (more set the overflow flag).
// They are sorted and deduplicated in shared memory, each is tested, and the hits are emitted in
// ascending (distance key, candidate) order, up to the query's max_hits: the order the reference's
// repeated minimum picks produce (scene_cast.wgsl:466-520). The grid is the one dyn_query builds from
// the current states just before (the reference's query run refreshes its AABBs and entries,
// crates/dynamis-rigid/src/integrate.rs:110-133).
//
// Hull colliders: the reference walks a hull's triangles through a BVH (scene.wgsl:363-401,
// 568-628); here they are walked in index order. A ray keeps the nearest triangle either way (the
// first in walk order at an exact tie); the sphere / point query's normal, which the reference takes
// from the first penetrating triangle of its walk (below), can name another face.
#pragma once

#include "narrow.cuh"
#include "step.cuh"

namespace dyn {

constexpr uint32_t kQueryThreads = 128u;
constexpr uint32_t kGridWalkCells = 4096u;  // GRID_WALK_CELLS, grid_index.wgsl:6
constexpr float kQNoHit = 3.402823466e38f;

struct QHit {
    float distance;
    f3 point, normal;
    uint32_t triangle;
};
__device__ __forceinline__ QHit q_no_hit() { return QHit{kQNoHit, s3(0.0f), s3(0.0f), DYN_NO_TRIANGLE}; }
__device__ __forceinline__ QHit q_nearest(const QHit& held, const QHit& candidate) {
    return candidate.distance < held.distance ? candidate : held;
}

// ---- rays (scene.wgsl:10-218, 259-285) ----
__device__ QHit ray_sphere(f3 origin, f3 direction, float extent, f3 center, float radius) {
    const f3 offset = origin - center;
    const float quadratic = dot(direction, direction);
    const float linear = dot(offset, direction);
    const float constant = dot(offset, offset) - radius * radius;
    const float discriminant = linear * linear - quadratic * constant;
    if (quadratic <= 0.0f || discriminant < 0.0f) return q_no_hit();
    const float root = sqrtf(discriminant);
    float t = (-linear - root) / quadratic;
    if (t < 0.0f) t = (-linear + root) / quadratic;
    if (t < 0.0f || t > extent) return q_no_hit();
    const f3 point = origin + direction * t;
    return QHit{t, point, normalize(point - center), DYN_NO_TRIANGLE};
}

__device__ QHit ray_box(f3 origin, f3 direction, float extent, f3 center, float4 q, f3 half_extents) {
    const float4 qc = quat_conj(q);
    const f3 lo = quat_rotate(qc, origin - center);
    const f3 ld = quat_rotate(qc, direction);
    const f3 inv = mk3(1.0f / ld.x, 1.0f / ld.y, 1.0f / ld.z);
    float tmin = 0.0f, tmax = extent;
    f3 normal_axis = s3(0.0f);
    for (uint32_t axis = 0; axis < 3u; ++axis) {
        const float o = comp(lo, axis);
        const f3 n = axis == 0u ? mk3(1.0f, 0.0f, 0.0f) : (axis == 1u ? mk3(0.0f, 1.0f, 0.0f) : mk3(0.0f, 0.0f, 1.0f));
        const float half = comp(half_extents, axis);
        float t1 = (-half - o) * comp(inv, axis);
        float t2 = (half - o) * comp(inv, axis);
        f3 candidate = n;
        if (t1 > t2) {
            const float tmp = t1;
            t1 = t2;
            t2 = tmp;
            candidate = -n;
        }
        if (t1 > tmin) {
            tmin = t1;
            normal_axis = candidate;
        }
        if (t2 < tmax) tmax = t2;
        if (tmin > tmax) return q_no_hit();
    }
    if (tmin < 0.0f || tmin > extent) return q_no_hit();
    const f3 local_point = lo + ld * tmin;
    return QHit{tmin, center + quat_rotate(q, local_point), quat_rotate(q, normal_axis), DYN_NO_TRIANGLE};
}

__device__ __forceinline__ float ray_quadratic_root(float quadratic, float linear, float constant) {
    const float discriminant = linear * linear - quadratic * constant;
    if (quadratic <= 0.0f || discriminant < 0.0f) return kQNoHit;
    const float root = sqrtf(discriminant);
    const float near = (-linear - root) / quadratic;
    if (near >= 0.0f) return near;
    const float far = (-linear + root) / quadratic;
    if (far >= 0.0f) return far;
    return kQNoHit;
}

__device__ QHit ray_sphere_candidate(f3 origin, f3 direction, float extent, f3 center, float radius, f3 hemisphere) {
    const f3 offset = origin - center;
    const float t = ray_quadratic_root(dot(direction, direction), dot(offset, direction), dot(offset, offset) - radius * radius);
    if (t == kQNoHit || t > extent) return q_no_hit();
    const f3 local = offset + direction * t;
    if (length(hemisphere) > 0.0f && dot(local, hemisphere) < 0.0f) return q_no_hit();
    return QHit{t, origin + direction * t, sign_normalize(local), DYN_NO_TRIANGLE};
}

__device__ QHit ray_swept_segment(f3 origin, f3 direction, float extent, f3 start, f3 end, float radius) {
    const f3 basis = end - start;
    const float basis_squared = dot(basis, basis);
    if (basis_squared <= 0.0f) return ray_sphere_candidate(origin, direction, extent, start, radius, s3(0.0f));
    const f3 offset = origin - start;
    const float axial_offset = dot(basis, offset);
    const float axial_direction = dot(basis, direction);
    const float inverse_basis = 1.0f / basis_squared;
    const f3 perp_offset = offset - basis * (axial_offset * inverse_basis);
    const f3 perp_direction = direction - basis * (axial_direction * inverse_basis);
    QHit best = q_no_hit();
    const float side = ray_quadratic_root(dot(perp_direction, perp_direction), dot(perp_offset, perp_direction),
                                          dot(perp_offset, perp_offset) - radius * radius);
    if (side != kQNoHit && side <= extent) {
        const float axial = axial_offset + side * axial_direction;
        if (axial >= 0.0f && axial <= basis_squared) {
            const f3 normal = sign_normalize(perp_offset + perp_direction * side);
            best = q_nearest(best, QHit{side, origin + direction * side, normal, DYN_NO_TRIANGLE});
        }
    }
    best = q_nearest(best, ray_sphere_candidate(origin, direction, extent, start, radius, -basis));
    best = q_nearest(best, ray_sphere_candidate(origin, direction, extent, end, radius, basis));
    return best;
}

__device__ __forceinline__ QHit ray_capsule(f3 origin, f3 direction, float extent, f3 center, f3 axis, float half_height,
                                            float radius) {
    return ray_swept_segment(origin, direction, extent, center - axis * half_height, center + axis * half_height, radius);
}

__device__ QHit ray_disc(f3 origin, f3 direction, float extent, f3 center, f3 axis, float radius_squared) {
    const float travel = dot(direction, axis);
    if (fabsf(travel) < 1e-8f) return q_no_hit();
    const float t = dot(center - origin, axis) / travel;
    if (t < 0.0f || t > extent) return q_no_hit();
    const f3 local = origin + direction * t - center;
    if (dot(local, local) > radius_squared) return q_no_hit();
    return QHit{t, origin + direction * t, travel < 0.0f ? axis : -axis, DYN_NO_TRIANGLE};
}

__device__ QHit ray_cylinder(f3 origin, f3 direction, float extent, f3 center, f3 axis, float half_height, float radius) {
    const f3 start = center - axis * half_height;
    const f3 end = center + axis * half_height;
    const f3 basis = end - start;
    const float basis_squared = dot(basis, basis);
    const float radius_squared = radius * radius;
    if (basis_squared <= 0.0f) return ray_disc(origin, direction, extent, center, axis, radius_squared);
    const f3 offset = origin - start;
    const float axial_offset = dot(basis, offset);
    const float axial_direction = dot(basis, direction);
    QHit best = q_no_hit();
    const float inverse_basis = 1.0f / basis_squared;
    const f3 perp_offset = offset - basis * (axial_offset * inverse_basis);
    const f3 perp_direction = direction - basis * (axial_direction * inverse_basis);
    const float side = ray_quadratic_root(dot(perp_direction, perp_direction), dot(perp_offset, perp_direction),
                                          dot(perp_offset, perp_offset) - radius_squared);
    if (side != kQNoHit && side <= extent) {
        const float axial = axial_offset + side * axial_direction;
        if (axial >= 0.0f && axial <= basis_squared) {
            const f3 normal = sign_normalize(perp_offset + perp_direction * side);
            best = q_nearest(best, QHit{side, origin + direction * side, normal, DYN_NO_TRIANGLE});
        }
    }
    if (fabsf(axial_direction) > 0.0f) {
        for (uint32_t cap = 0; cap < 2u; ++cap) {
            const float cap_at = cap == 1u ? basis_squared - axial_offset : axial_offset;
            const float t = cap_at / (cap == 1u ? axial_direction : -axial_direction);
            if (t < 0.0f || t > extent) continue;
            const f3 local = offset + direction * t - basis * (cap == 1u ? 1.0f : 0.0f);
            if (dot(local, local) <= radius_squared) {
                const f3 normal = sign_normalize(cap == 1u ? basis : -basis);
                best = q_nearest(best, QHit{t, origin + direction * t, normal, DYN_NO_TRIANGLE});
            }
        }
    }
    return best;
}

__device__ QHit ray_triangle(f3 origin, f3 direction, float extent, f3 a, f3 b, f3 c) {
    const f3 edge1 = b - a;
    const f3 edge2 = c - a;
    const f3 p = cross(direction, edge2);
    const float det = dot(edge1, p);
    if (fabsf(det) < 1e-8f) return q_no_hit();
    const float inv_det = 1.0f / det;
    const f3 t_vec = origin - a;
    const float u = dot(t_vec, p) * inv_det;
    if (u < 0.0f || u > 1.0f) return q_no_hit();
    const f3 qv = cross(t_vec, edge1);
    const float v = dot(direction, qv) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return q_no_hit();
    const float t = dot(edge2, qv) * inv_det;
    if (t < 0.0f || t > extent) return q_no_hit();
    const f3 normal = sign_normalize(cross(edge1, edge2));
    return QHit{t, origin + direction * t, det < 0.0f ? -normal : normal, DYN_NO_TRIANGLE};
}

__device__ __forceinline__ f3 hull_corner(const DeviceWorld& w, const dyn_shape_source_record& src, uint32_t corner, f3 scale) {
    return xyz(w.vertices[src.vertex_offset + corner]) * scale;
}

// ray_scene (scene.wgsl:306-320) of a hull: the nearest triangle in the hull's own frame.
__device__ QHit ray_hull(const DeviceWorld& w, const WShape& s, f3 origin, f3 direction, float extent) {
    const float4 qc = quat_conj(s.rotation);
    const f3 lo = quat_rotate(qc, origin - s.center);
    const f3 ld = quat_rotate(qc, direction);
    const dyn_shape_source_record& src = w.sources[s.source];
    const uint2 range = w.hull_tri_range[s.source];
    QHit best = q_no_hit();
    for (uint32_t t = 0; t < range.y; ++t) {
        const uint4 tri = w.hull_tris[range.x + t];
        QHit hit = ray_triangle(lo, ld, extent, hull_corner(w, src, tri.x, s.scale), hull_corner(w, src, tri.y, s.scale),
                                hull_corner(w, src, tri.z, s.scale));
        if (hit.distance != kQNoHit) hit.triangle = t;
        if (hit.distance < best.distance) best = hit;
    }
    if (best.distance == kQNoHit) return best;
    best.point = s.center + quat_rotate(s.rotation, best.point);
    best.normal = sign_normalize(quat_rotate(s.rotation, best.normal));
    return best;
}

__device__ __forceinline__ f3 shape_axis(const WShape& s) { return quat_rotate(s.rotation, mk3(0.0f, 1.0f, 0.0f)); }

// shape_ray (scene.wgsl:813-872)
__device__ QHit shape_ray(const DeviceWorld& w, const WShape& s, f3 origin, f3 direction, float extent) {
    const f3 heading = normalize(direction);
    if (s.kind == DYN_SHAPE_PLANE) {
        const f3 normal = shape_axis(s);
        const float travel = dot(heading, normal);
        if (fabsf(travel) < 1e-8f) return q_no_hit();
        const float t = dot(s.center - origin, normal) / travel;
        if (t < 0.0f || t > extent) return q_no_hit();
        return QHit{t, origin + heading * t, normal, DYN_NO_TRIANGLE};
    }
    if (shape_has_source(s.kind)) return ray_hull(w, s, origin, heading, extent);
    const bool unscaled = s.scale.x == 1.0f && s.scale.y == 1.0f && s.scale.z == 1.0f;
    if (unscaled) {
        if (s.kind == DYN_SHAPE_SPHERE) return ray_sphere(origin, heading, extent, s.center, s.radius);
        if (s.kind == DYN_SHAPE_CUBOID) return ray_box(origin, heading, extent, s.center, s.rotation, s.half_extents);
        if (s.kind == DYN_SHAPE_CAPSULE) return ray_capsule(origin, heading, extent, s.center, shape_axis(s), s.half_height, s.radius);
        if (s.kind == DYN_SHAPE_CYLINDER) return ray_cylinder(origin, heading, extent, s.center, shape_axis(s), s.half_height, s.radius);
        return q_no_hit();
    }
    const float4 inv_rotation = quat_conj(s.rotation);
    const f3 unscale = mk3(1.0f / s.scale.x, 1.0f / s.scale.y, 1.0f / s.scale.z);
    const f3 lo = quat_rotate(inv_rotation, origin - s.center) * unscale;
    const f3 ld = quat_rotate(inv_rotation, heading) * unscale;
    const float local_extent = extent * length(ld);
    QHit local;
    if (s.kind == DYN_SHAPE_SPHERE) {
        local = ray_sphere(lo, ld, local_extent, s3(0.0f), s.radius);
    } else if (s.kind == DYN_SHAPE_CAPSULE) {
        local = ray_capsule(lo, ld, local_extent, s3(0.0f), mk3(0.0f, 1.0f, 0.0f), s.half_height, s.radius);
    } else if (s.kind == DYN_SHAPE_CYLINDER) {
        local = ray_cylinder(lo, ld, local_extent, s3(0.0f), mk3(0.0f, 1.0f, 0.0f), s.half_height, s.radius);
    } else {
        return q_no_hit();  // a scaled cuboid answers no ray here, as in the reference
    }
    if (local.distance == kQNoHit) return q_no_hit();
    QHit hit;
    hit.distance = local.distance;
    hit.triangle = DYN_NO_TRIANGLE;
    hit.point = s.center + quat_rotate(s.rotation, (lo + ld * local.distance) * s.scale);
    hit.normal = quat_rotate(s.rotation, sign_normalize(local.normal * unscale));
    return hit;
}

// ---- the query's own shape and its tests (scene_cast.wgsl:136-196, 365-432) ----
__device__ __forceinline__ WShape query_shape(const dyn_query_record& q, f3 center) {
    WShape s;
    s.kind = q.shape_kind;
    s.radius = q.radius;
    s.half_height = q.half_height;
    s.center = center;
    s.half_extents = mk3(q.half_extents[0], q.half_extents[1], q.half_extents[2]);
    s.rotation = make_float4(q.orientation[0], q.orientation[1], q.orientation[2], q.orientation[3]);
    s.source = q.source;
    s.scale = s3(1.0f);
    return s;
}
// The shape a query tests with. QueryRecord::sphere, ::point and ::cuboid leave the orientation zero
// (crates/dynamis-abi/src/query.rs:115-144 over a zeroed record), and a zero quaternion rotates every
// support offset to nothing, so the reference's probe answers with its centre point (the
// normalisation of the zero direction that precedes it is left to the backend: here it is skipped,
// and the probe is that point). The query's box (query_box) keeps the record's own shape.
__device__ __forceinline__ WShape query_probe(const dyn_query_record& q, f3 center) {
    WShape s = query_shape(q, center);
    if (s.rotation.x == 0.0f && s.rotation.y == 0.0f && s.rotation.z == 0.0f && s.rotation.w == 0.0f) {
        s.kind = DYN_SHAPE_SPHERE;
        s.radius = 0.0f;
        s.rotation = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    }
    return s;
}
__device__ __forceinline__ f3 q_origin(const dyn_query_record& q) { return mk3(q.origin[0], q.origin[1], q.origin[2]); }
__device__ __forceinline__ f3 q_direction(const dyn_query_record& q) {
    return mk3(q.direction[0], q.direction[1], q.direction[2]);
}

// convex.wgsl:627-630: convex_hit with the normal turned to face the probe
__device__ __forceinline__ Hit penetration_hit(const DeviceWorld& w, const WShape& probe, const WShape& solid) {
    Hit h = convex_hit(w, probe, solid);
    h.normal = -h.normal;
    return h;
}

// scene.wgsl:536-555 for one hull triangle in the hull's frame
struct QClosest {
    float distance;
    f3 normal;
    bool penetrating;
};
__device__ QClosest plane_distance(const DeviceWorld& w, const dyn_shape_source_record& src, uint4 tri, f3 scale,
                                   const WShape& local) {
    const f3 a = hull_corner(w, src, tri.x, scale), b = hull_corner(w, src, tri.y, scale), c = hull_corner(w, src, tri.z, scale);
    f3 n = sign_normalize(cross(b - a, c - a));
    float offset = dot(local.center - a, n);
    if (offset < 0.0f) {
        n = -n;
        offset = -offset;
    }
    const f3 deep = support(w, local, -n);
    const float extent = dot(deep - local.center, -n);
    const float separation = offset - extent;
    return QClosest{separation, n, separation < 0.0f};
}

// overlap_world_geom (scene_cast.wgsl:180-194): its separation for a plane; for any other collider
// only the normal it leaves behind, which is what a sphere or point query reports (the reference
// evaluates both arms of its select, scene_cast.wgsl:402-406, this one last): (0, 1, 0) for an
// analytic shape (scene.wgsl:568-578), the closest hull triangle's normal for a hull, where the first
// penetrating triangle stops the walk (scene.wgsl:630-648).
__device__ float overlap_world_geom(const DeviceWorld& w, const dyn_query_record& q, const WShape& scene, f3* out_normal) {
    if (scene.kind == DYN_SHAPE_PLANE) {
        const f3 n = shape_axis(scene);
        *out_normal = n;
        return dot(q_origin(q) - scene.center, n) - q.extent;
    }
    f3 normal = mk3(0.0f, 1.0f, 0.0f);
    float distance = kQNoHit;
    if (shape_has_source(scene.kind)) {
        const float4 qc = quat_conj(scene.rotation);
        WShape local = query_probe(q, quat_rotate(qc, q_origin(q) - scene.center));
        local.rotation = quat_mul(qc, local.rotation);
        const dyn_shape_source_record& src = w.sources[scene.source];
        const uint2 range = w.hull_tri_range[scene.source];
        bool found = false;
        for (uint32_t t = 0; t < range.y; ++t) {
            const QClosest c = plane_distance(w, src, w.hull_tris[range.x + t], scene.scale, local);
            if (c.penetrating || c.distance < distance) {
                distance = c.distance;
                normal = c.normal;
                found = true;
                if (c.penetrating) break;
            }
        }
        if (found) normal = sign_normalize(quat_rotate(scene.rotation, normal));
    }
    *out_normal = normal;
    return distance;
}

// overlap_hit (scene_cast.wgsl:160-178)
__device__ float overlap_hit(const DeviceWorld& w, const dyn_query_record& q, const WShape& world, f3* out_normal) {
    WShape probe = query_probe(q, q_origin(q));
    probe.radius = 0.0f;
    const GjkOut closest = gjk_phase(w, probe, world);
    if (closest.pen) {
        const Hit hit = penetration_hit(w, query_probe(q, q_origin(q)), world);
        *out_normal = hit.normal;
        return -q.extent + wmax(hit.distance + q.extent, 0.0f);
    }
    if (closest.dist <= q.extent) {
        *out_normal = -closest.normal;
        return closest.dist - q.extent;
    }
    return kQNoHit;
}

// shape_sweep (scene.wgsl:219-257) of the query's shape against a collider
__device__ QHit shape_sweep(const DeviceWorld& w, const WShape& moving, const WShape& target, f3 start, f3 direction,
                            float max_dist) {
    const f3 heading = normalize(direction);
    if (target.kind == DYN_SHAPE_PLANE) {
        const f3 normal = shape_axis(target);
        const float travel = dot(heading, normal);
        if (travel >= 0.0f) return q_no_hit();
        const float extent = dot(support(w, moving, -normal) - moving.center, -normal);
        const float offset = dot(start - target.center, normal);
        const float time = wmax((offset - extent) / (-travel), 0.0f);
        if (time > max_dist) return q_no_hit();
        return QHit{time, start + heading * time, normal, DYN_NO_TRIANGLE};
    }
    WShape moved = moving;
    float time = 0.0f;
    f3 normal = sign_normalize(moving.center - target.center);
    for (uint32_t iteration = 0; iteration < 8u; ++iteration) {
        moved.center = start + heading * time;
        const GjkOut closest = gjk_phase(w, moved, target);
        if (closest.pen || closest.dist < 1e-4f) return QHit{time, start + heading * time, normal, DYN_NO_TRIANGLE};
        normal = -closest.normal;
        time = time + closest.dist;
        if (time > max_dist) return q_no_hit();
    }
    return q_no_hit();
}

// resolve_hit (scene_cast.wgsl:384-432) of one collider
__device__ QHit resolve_hit(const DeviceWorld& w, const dyn_query_record& q, const WShape& world) {
    const uint32_t kind = q.kind;
    if (kind == DYN_QUERY_RAY) {
        const f3 direction = normalize(q_direction(q));
        QHit hit = shape_ray(w, world, q_origin(q), direction, q.extent);
        if (hit.distance == kQNoHit) return hit;
        if (dot(hit.normal, direction) > 0.0f) hit.normal = -hit.normal;
        return hit;
    }
    const bool world_geom = shape_world_geometry(world.kind);
    if (kind == DYN_QUERY_SWEEP) {
        const QHit hit = shape_sweep(w, query_probe(q, q_origin(q)), world, q_origin(q), q_direction(q), q.extent);
        return hit.distance < kQNoHit ? hit : q_no_hit();
    }
    f3 normal = s3(0.0f);
    if (kind == DYN_QUERY_SPHERE || kind == DYN_QUERY_POINT) {
        const float from_hit = overlap_hit(w, q, world, &normal);
        const float from_geom = overlap_world_geom(w, q, world, &normal);
        const float separation = world_geom ? from_geom : from_hit;
        if (separation < kQNoHit) return QHit{separation, world.center, normal, DYN_NO_TRIANGLE};
        return q_no_hit();
    }
    if (world_geom) {
        const float separation = overlap_world_geom(w, q, world, &normal);
        if (separation < kQNoHit) return QHit{separation, world.center, normal, DYN_NO_TRIANGLE};
        return q_no_hit();
    }
    const WShape probe = query_probe(q, q_origin(q));
    const GjkOut closest = gjk_phase(w, probe, world);
    if (closest.pen) {
        const Hit hit = penetration_hit(w, probe, world);
        return QHit{hit.distance, (closest.pa + closest.pb) * 0.5f, hit.normal, DYN_NO_TRIANGLE};
    }
    return q_no_hit();
}

// body_passes (scene_cast.wgsl:196-222) and collider_filter_query (core.wgsl:285-291)
__device__ bool query_passes(const DeviceWorld& w, const dyn_query_record& q, uint32_t slot) {
    const uint32_t row = w.c_owner[slot];
    if (row == DYN_NO_BODY) return false;
    const uint4 ident = w.ident[row];  // body_id, generation, group, mask
    const dyn_query_filter_record& f = q.filters;
    if (f.exclude_id != DYN_NO_BODY && ident.x == f.exclude_id && ident.y == f.exclude_generation) return false;
    if (f.include_id != DYN_NO_BODY && (ident.x != f.include_id || ident.y != f.include_generation)) return false;
    const uint4 kind = w.c_kind[slot];  // kind, flags, source
    const BodyHot& h = w.hot[row];
    if ((f.flags & DYN_FILTER_IGNORE_SENSORS) && (kind.y & DYN_COLLIDER_SENSOR)) return false;
    if ((f.flags & DYN_FILTER_IGNORE_SLEEPING) && h.aux.x != 0u) return false;
    if ((f.flags & DYN_FILTER_IGNORE_STATIC) && !moves(h.pos.w, h.aux.y)) return false;
    if ((f.flags & DYN_FILTER_IGNORE_KINEMATIC) && moves(h.pos.w, h.aux.y) && !simulates(h.pos.w, h.aux.y)) return false;
    if (f.group != 0u) {
        const uint2 cf = w.c_filter[slot];
        const uint32_t group = cf.x != DYN_NO_COLLISION_FILTER ? cf.x : ident.z;
        const uint32_t mask = cf.y != DYN_NO_COLLISION_FILTER ? cf.y : ident.w;
        if (!((f.group & mask) != 0u && (group & f.mask) != 0u)) return false;
    }
    return kind.x != DYN_SHAPE_NONE;
}

// query_world_aabb (scene_cast.wgsl:341-362)
__device__ DAabb query_box(const DeviceWorld& w, const dyn_query_record& q) {
    const f3 origin = q_origin(q);
    if (q.kind == DYN_QUERY_RAY) {
        const f3 direction = normalize(q_direction(q));
        const f3 end = origin + direction * q.extent;
        return DAabb{vmin(origin, end), vmax(origin, end)};
    }
    if (q.kind == DYN_QUERY_SWEEP) {
        DAabb a = world_aabb(w, query_shape(q, origin));
        const f3 direction = normalize(q_direction(q));
        const DAabb b = world_aabb(w, query_shape(q, origin + direction * q.extent));
        return DAabb{vmin(a.min, b.min), vmax(a.max, b.max)};
    }
    return world_aabb(w, query_shape(q, origin));
}

__device__ __forceinline__ uint32_t hit_key(float distance) {
    const uint32_t bits = __float_as_uint(distance);
    return (bits & 0x80000000u) != 0u ? ~bits : (bits | 0x80000000u);
}

// Bitonic sort of `width` (a power of two) values in shared memory, ascending, by the whole block.
template <typename T>
__device__ void block_bitonic(T* values, uint32_t width) {
    for (uint32_t k = 2u; k <= width; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0u; j >>= 1) {
            for (uint32_t index = threadIdx.x; index < width; index += blockDim.x) {
                const uint32_t other = index ^ j;
                if (other > index) {
                    const bool ascending = (index & k) == 0u;
                    const T a = values[index], b = values[other];
                    if (ascending ? a > b : a < b) {
                        values[index] = b;
                        values[other] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}

struct QueryShared {
    uint32_t candidates[DYN_QUERY_CANDIDATES];
    unsigned long long keys[DYN_QUERY_CANDIDATES];
    uint32_t candidate_count;
    uint32_t overflow;
    uint32_t hit_total;
};

__device__ __forceinline__ void push_candidate(QueryShared& sh, uint32_t slot) {
    const uint32_t at = atomicAdd(&sh.candidate_count, 1u);
    if (at >= DYN_QUERY_CANDIDATES) {
        sh.overflow = 1u;
        return;
    }
    sh.candidates[at] = slot;
}

// One block per query (scene_cast.wgsl:434-533).
__global__ void __launch_bounds__(kQueryThreads) k_scene_query(DeviceWorld w, dyn_query_record* queries,
                                                               dyn_query_hit_record* hits, uint32_t count) {
    extern __shared__ __align__(16) unsigned char smem[];
    QueryShared& sh = *reinterpret_cast<QueryShared*>(smem);
    for (uint32_t qi = blockIdx.x; qi < count; qi += gridDim.x) {
        const dyn_query_record q = queries[qi];
        if (threadIdx.x == 0) {
            sh.candidate_count = 0u;
            sh.overflow = 0u;
            sh.hit_total = 0u;
        }
        __syncthreads();
        // the candidates: entries of the cells the query's box covers, level by level
        const DAabb box = query_box(w, q);
        const uint32_t live = min(w.ctl[CTL_ENTRIES], w.e_cap);
        const float grid = base_cell(w);
        const uint32_t bits = cell_table_bits(w, live);
        const bool table_overflow = w.ctl[CTL_CELL_OVERFLOW] != 0u;
        const bool wants_colliders = (q.filters.targets & DYN_QUERY_TARGET_COLLIDERS) != 0u;
        uint32_t occupied = wants_colliders ? (w.counters[DYN_COUNTER_GRID_LEVELS] | w.counters[DYN_COUNTER_RESTING_LEVELS] |
                                                       w.counters[DYN_COUNTER_IMMOVABLE_LEVELS]) : 0u;
        while (occupied != 0u) {
            const uint32_t level = (uint32_t)__ffs(occupied) - 1u;
            occupied &= occupied - 1u;
            const float cs = level_size(level, grid);
            const I3 lo = floor_div(box.min, cs), hi = floor_div(box.max, cs);
            const long long sx = (long long)hi.x - lo.x + 1, sy = (long long)hi.y - lo.y + 1, sz = (long long)hi.z - lo.z + 1;
            const long long cells = sx * sy * sz;
            if (cells <= 0) continue;
            if (cells > (long long)kGridWalkCells) {
                // the whole level, its entries tested against the box
                const uint32_t first = lower_bound(w.ekey, live, level << DYN_LEVEL_KEY_SHIFT);
                const uint32_t end = lower_bound(w.ekey, live, (level + 1u) << DYN_LEVEL_KEY_SHIFT);
                for (uint32_t j = first + threadIdx.x; j < end && sh.candidate_count <= DYN_QUERY_CANDIDATES; j += blockDim.x) {
                    const GEntry e = load_entry(w, w.eval[j]);
                    if (!(e.mn.x <= box.max.x && e.mn.y <= box.max.y && e.mn.z <= box.max.z && box.min.x <= e.mx.x &&
                          box.min.y <= e.mx.y && box.min.z <= e.mx.z))
                        continue;
                    push_candidate(sh, e.info & DYN_ENTRY_INDEX_MASK);
                }
            } else {
                for (uint32_t c = threadIdx.x; c < (uint32_t)cells; c += blockDim.x) {
                    const uint32_t rows = (uint32_t)(sy * sz);
                    const I3 cell = I3{lo.x + (int)(c / rows), lo.y + (int)((c / (uint32_t)sz) % (uint32_t)sy), lo.z + (int)(c % (uint32_t)sz)};
                    const uint32_t key = cell_key(level, cell);
                    for (uint32_t j = cell_find(w, live, bits, table_overflow, key); j < live && w.ekey[j] == key; ++j) {
                        const GEntry e = load_entry(w, w.eval[j]);
                        push_candidate(sh, e.info & DYN_ENTRY_INDEX_MASK);
                    }
                }
            }
        }
        __syncthreads();
        // sorted, duplicates marked (an entry per covered cell of a collider)
        const uint32_t total = min(sh.candidate_count, DYN_QUERY_CANDIDATES);
        uint32_t width = 1u;
        while (width < total) width <<= 1;
        for (uint32_t i = threadIdx.x; i < width; i += blockDim.x) {
            if (i >= total) sh.candidates[i] = 0xFFFFFFFFu;
        }
        __syncthreads();
        block_bitonic(sh.candidates, width);
        // each distinct candidate's hit, keyed by (distance key, candidate)
        for (uint32_t i = threadIdx.x; i < width; i += blockDim.x) {
            unsigned long long key = ~0ull;
            if (i < total && !(i > 0u && sh.candidates[i] == sh.candidates[i - 1u])) {
                const uint32_t slot = sh.candidates[i];
                if (query_passes(w, q, slot)) {
                    const uint32_t row = w.c_owner[slot];
                    const DBody b = load_dbody(w.hot, row);
                    const QHit hit = resolve_hit(w, q, world_shape(b.position, b.orientation, load_dcoll(w, slot)));
                    if (hit.distance < kQNoHit) {
                        key = ((unsigned long long)hit_key(hit.distance) << 32) | slot;
                        atomicAdd(&sh.hit_total, 1u);
                    }
                }
            }
            sh.keys[i] = key;
        }
        __syncthreads();
        block_bitonic(sh.keys, width);
        const uint32_t capacity = min(q.max_hits, DYN_QUERY_CANDIDATES);
        const uint32_t emitted = min(capacity, sh.hit_total);
        for (uint32_t i = threadIdx.x; i < emitted; i += blockDim.x) {
            const uint32_t slot = (uint32_t)(sh.keys[i] & 0xFFFFFFFFull);
            const uint32_t row = w.c_owner[slot];
            const DBody b = load_dbody(w.hot, row);
            const QHit hit = resolve_hit(w, q, world_shape(b.position, b.orientation, load_dcoll(w, slot)));
            const uint4 ident = w.ident[row];
            dyn_query_hit_record r;
            r.body_id = ident.x;
            r.body_generation = ident.y;
            r.distance = hit.distance;
            r.scene_target = (DYN_ENTRY_KIND_COLLIDER << DYN_ENTRY_KIND_SHIFT) | slot;
            r.point[0] = hit.point.x;
            r.point[1] = hit.point.y;
            r.point[2] = hit.point.z;
            r.triangle = hit.triangle;
            r.normal[0] = hit.normal.x;
            r.normal[1] = hit.normal.y;
            r.normal[2] = hit.normal.z;
            r.surface = DYN_NO_SURFACE;  // hull triangles carry no surface (crates/dynamis-world/src/shape_pool.rs:557-580)
            hits[q.hit_base + i] = r;
        }
        if (threadIdx.x == 0) {
            queries[qi].count = emitted;
            queries[qi].overflow = (sh.overflow != 0u || emitted < sh.hit_total) ? 1u : 0u;
        }
        __syncthreads();
    }
}

}  // namespace dyn
