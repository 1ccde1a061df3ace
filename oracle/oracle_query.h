// oracle_query.h - the scene-query tests restated on the CPU (test infrastructure: the checker of
// dyn_query, never part of the library). Every function follows the WGSL it cites, operand for
// operand: crates/dynamis-shader/shaders/scene.wgsl:1-258 (rays, sweeps), 259-320 (triangle rays),
// 536-660 (triangle closest), 813-873 (shape_ray); scene_cast.wgsl:136-432 (the query's shape, the
// overlap tests, the filters, the query box, resolve_hit). A hull's triangles are walked in index
// order (the reference walks them through a BVH).
#pragma once

#include <cstdint>
#include <vector>

#include "dynamis_abi.h"
#include "oracle_geom.h"

namespace orc {

struct HullTriangles {
    const uint32_t* tris = nullptr;    // index triples, hull by hull
    const uint32_t* ranges = nullptr;  // [source]: first triangle, triangle count
    uint32_t sources = 0;
};

inline ShapeHit q_no_hit() { return ShapeHit{kNoHit, splat3(0.0f), splat3(0.0f), DYN_NO_TRIANGLE}; }
inline ShapeHit q_nearest(const ShapeHit& held, const ShapeHit& candidate) {
    return candidate.distance < held.distance ? candidate : held;
}

inline ShapeHit ray_sphere(V3 origin, V3 direction, float extent, V3 center, float radius) {
    V3 offset = origin - center;
    float quadratic = dot(direction, direction);
    float linear = dot(offset, direction);
    float constant = dot(offset, offset) - radius * radius;
    float discriminant = linear * linear - quadratic * constant;
    if (quadratic <= 0.0f || discriminant < 0.0f) return q_no_hit();
    float root = std::sqrt(discriminant);
    float t = (-linear - root) / quadratic;
    if (t < 0.0f) t = (-linear + root) / quadratic;
    if (t < 0.0f || t > extent) return q_no_hit();
    V3 point = origin + direction * t;
    return ShapeHit{t, point, normalize(point - center), DYN_NO_TRIANGLE};
}

inline ShapeHit ray_box(V3 origin, V3 direction, float extent, V3 center, V4 q, V3 half_extents) {
    V4 qc = quat_conjugate(q);
    V3 lo = quat_rotate(qc, origin - center);
    V3 ld = quat_rotate(qc, direction);
    V3 inv = V3{1.0f / ld.x, 1.0f / ld.y, 1.0f / ld.z};
    float tmin = 0.0f, tmax = extent;
    V3 normal_axis = splat3(0.0f);
    for (uint32_t axis = 0; axis < 3u; ++axis) {
        float o = comp(lo, axis);
        V3 n = axis == 0u ? V3{1.0f, 0.0f, 0.0f} : (axis == 1u ? V3{0.0f, 1.0f, 0.0f} : V3{0.0f, 0.0f, 1.0f});
        float half = comp(half_extents, axis);
        float t1 = (-half - o) * comp(inv, axis);
        float t2 = (half - o) * comp(inv, axis);
        V3 candidate = n;
        if (t1 > t2) {
            float tmp = t1;
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
    V3 local_point = lo + ld * tmin;
    return ShapeHit{tmin, center + quat_rotate(q, local_point), quat_rotate(q, normal_axis), DYN_NO_TRIANGLE};
}

inline float ray_quadratic_root(float quadratic, float linear, float constant) {
    float discriminant = linear * linear - quadratic * constant;
    if (quadratic <= 0.0f || discriminant < 0.0f) return kNoHit;
    float root = std::sqrt(discriminant);
    float near_t = (-linear - root) / quadratic;
    if (near_t >= 0.0f) return near_t;
    float far_t = (-linear + root) / quadratic;
    if (far_t >= 0.0f) return far_t;
    return kNoHit;
}

inline ShapeHit ray_sphere_candidate(V3 origin, V3 direction, float extent, V3 center, float radius, V3 hemisphere) {
    V3 offset = origin - center;
    float t = ray_quadratic_root(dot(direction, direction), dot(offset, direction), dot(offset, offset) - radius * radius);
    if (t == kNoHit || t > extent) return q_no_hit();
    V3 local = offset + direction * t;
    if (length(hemisphere) > 0.0f && dot(local, hemisphere) < 0.0f) return q_no_hit();
    return ShapeHit{t, origin + direction * t, sign_normalize(local), DYN_NO_TRIANGLE};
}

inline ShapeHit ray_swept_segment(V3 origin, V3 direction, float extent, V3 start, V3 end, float radius) {
    V3 basis = end - start;
    float basis_squared = dot(basis, basis);
    if (basis_squared <= 0.0f) return ray_sphere_candidate(origin, direction, extent, start, radius, splat3(0.0f));
    V3 offset = origin - start;
    float axial_offset = dot(basis, offset);
    float axial_direction = dot(basis, direction);
    float inverse_basis = 1.0f / basis_squared;
    V3 perp_offset = offset - basis * (axial_offset * inverse_basis);
    V3 perp_direction = direction - basis * (axial_direction * inverse_basis);
    ShapeHit best = q_no_hit();
    float side = ray_quadratic_root(dot(perp_direction, perp_direction), dot(perp_offset, perp_direction),
                                    dot(perp_offset, perp_offset) - radius * radius);
    if (side != kNoHit && side <= extent) {
        float axial = axial_offset + side * axial_direction;
        if (axial >= 0.0f && axial <= basis_squared) {
            V3 normal = sign_normalize(perp_offset + perp_direction * side);
            best = q_nearest(best, ShapeHit{side, origin + direction * side, normal, DYN_NO_TRIANGLE});
        }
    }
    best = q_nearest(best, ray_sphere_candidate(origin, direction, extent, start, radius, -basis));
    best = q_nearest(best, ray_sphere_candidate(origin, direction, extent, end, radius, basis));
    return best;
}

inline ShapeHit ray_capsule(V3 origin, V3 direction, float extent, V3 center, V3 axis, float half_height, float radius) {
    return ray_swept_segment(origin, direction, extent, center - axis * half_height, center + axis * half_height, radius);
}

inline ShapeHit ray_disc(V3 origin, V3 direction, float extent, V3 center, V3 axis, float radius_squared) {
    float travel = dot(direction, axis);
    if (std::fabs(travel) < 1e-8f) return q_no_hit();
    float t = dot(center - origin, axis) / travel;
    if (t < 0.0f || t > extent) return q_no_hit();
    V3 local = origin + direction * t - center;
    if (dot(local, local) > radius_squared) return q_no_hit();
    return ShapeHit{t, origin + direction * t, travel < 0.0f ? axis : -axis, DYN_NO_TRIANGLE};
}

inline ShapeHit ray_cylinder(V3 origin, V3 direction, float extent, V3 center, V3 axis, float half_height, float radius) {
    V3 start = center - axis * half_height;
    V3 end = center + axis * half_height;
    V3 basis = end - start;
    float basis_squared = dot(basis, basis);
    float radius_squared = radius * radius;
    if (basis_squared <= 0.0f) return ray_disc(origin, direction, extent, center, axis, radius_squared);
    V3 offset = origin - start;
    float axial_offset = dot(basis, offset);
    float axial_direction = dot(basis, direction);
    ShapeHit best = q_no_hit();
    float inverse_basis = 1.0f / basis_squared;
    V3 perp_offset = offset - basis * (axial_offset * inverse_basis);
    V3 perp_direction = direction - basis * (axial_direction * inverse_basis);
    float side = ray_quadratic_root(dot(perp_direction, perp_direction), dot(perp_offset, perp_direction),
                                    dot(perp_offset, perp_offset) - radius_squared);
    if (side != kNoHit && side <= extent) {
        float axial = axial_offset + side * axial_direction;
        if (axial >= 0.0f && axial <= basis_squared) {
            V3 normal = sign_normalize(perp_offset + perp_direction * side);
            best = q_nearest(best, ShapeHit{side, origin + direction * side, normal, DYN_NO_TRIANGLE});
        }
    }
    if (std::fabs(axial_direction) > 0.0f) {
        for (uint32_t cap = 0; cap < 2u; ++cap) {
            float cap_at = cap == 1u ? basis_squared - axial_offset : axial_offset;
            float t = cap_at / (cap == 1u ? axial_direction : -axial_direction);
            if (t < 0.0f || t > extent) continue;
            V3 local = offset + direction * t - basis * (cap == 1u ? 1.0f : 0.0f);
            if (dot(local, local) <= radius_squared) {
                V3 normal = sign_normalize(cap == 1u ? basis : -basis);
                best = q_nearest(best, ShapeHit{t, origin + direction * t, normal, DYN_NO_TRIANGLE});
            }
        }
    }
    return best;
}

inline ShapeHit ray_triangle(V3 origin, V3 direction, float extent, V3 a, V3 b, V3 c) {
    V3 edge1 = b - a;
    V3 edge2 = c - a;
    V3 p = cross(direction, edge2);
    float det = dot(edge1, p);
    if (std::fabs(det) < 1e-8f) return q_no_hit();
    float inv_det = 1.0f / det;
    V3 t_vec = origin - a;
    float u = dot(t_vec, p) * inv_det;
    if (u < 0.0f || u > 1.0f) return q_no_hit();
    V3 qv = cross(t_vec, edge1);
    float v = dot(direction, qv) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return q_no_hit();
    float t = dot(edge2, qv) * inv_det;
    if (t < 0.0f || t > extent) return q_no_hit();
    V3 normal = sign_normalize(cross(edge1, edge2));
    return ShapeHit{t, origin + direction * t, det < 0.0f ? -normal : normal, DYN_NO_TRIANGLE};
}

inline V3 hull_corner(const Shapes& sh, const dyn_shape_source_record& src, uint32_t corner, V3 scale) {
    return xyz(sh.vertices[src.vertex_offset + corner]) * scale;
}

inline ShapeHit ray_hull(const Shapes& sh, const HullTriangles& ht, const WorldShape& s, V3 origin, V3 direction,
                         float extent) {
    V4 qc = quat_conjugate(s.rotation);
    V3 lo = quat_rotate(qc, origin - s.center);
    V3 ld = quat_rotate(qc, direction);
    const dyn_shape_source_record& src = sh.sources[s.source];
    uint32_t first = ht.ranges[2 * s.source], count = ht.ranges[2 * s.source + 1];
    ShapeHit best = q_no_hit();
    for (uint32_t t = 0; t < count; ++t) {
        const uint32_t* tri = ht.tris + 3 * (size_t)(first + t);
        ShapeHit hit = ray_triangle(lo, ld, extent, hull_corner(sh, src, tri[0], s.scale), hull_corner(sh, src, tri[1], s.scale),
                                    hull_corner(sh, src, tri[2], s.scale));
        if (hit.distance != kNoHit) hit.triangle = t;
        if (hit.distance < best.distance) best = hit;
    }
    if (best.distance == kNoHit) return best;
    best.point = s.center + quat_rotate(s.rotation, best.point);
    best.normal = sign_normalize(quat_rotate(s.rotation, best.normal));
    return best;
}

inline ShapeHit shape_ray(const Shapes& sh, const HullTriangles& ht, const WorldShape& s, V3 origin, V3 direction,
                          float extent) {
    V3 heading = normalize(direction);
    if (s.kind == DYN_SHAPE_PLANE) {
        V3 normal = shape_axis(s);
        float travel = dot(heading, normal);
        if (std::fabs(travel) < 1e-8f) return q_no_hit();
        float t = dot(s.center - origin, normal) / travel;
        if (t < 0.0f || t > extent) return q_no_hit();
        return ShapeHit{t, origin + heading * t, normal, DYN_NO_TRIANGLE};
    }
    if (shape_source(s.kind)) return ray_hull(sh, ht, s, origin, heading, extent);
    bool unscaled = s.scale.x == 1.0f && s.scale.y == 1.0f && s.scale.z == 1.0f;
    if (unscaled) {
        if (s.kind == DYN_SHAPE_SPHERE) return ray_sphere(origin, heading, extent, s.center, s.radius);
        if (s.kind == DYN_SHAPE_CUBOID) return ray_box(origin, heading, extent, s.center, s.rotation, s.half_extents);
        if (s.kind == DYN_SHAPE_CAPSULE) return ray_capsule(origin, heading, extent, s.center, shape_axis(s), s.half_height, s.radius);
        if (s.kind == DYN_SHAPE_CYLINDER) return ray_cylinder(origin, heading, extent, s.center, shape_axis(s), s.half_height, s.radius);
        return q_no_hit();
    }
    V4 inv_rotation = quat_conjugate(s.rotation);
    V3 unscale = V3{1.0f / s.scale.x, 1.0f / s.scale.y, 1.0f / s.scale.z};
    V3 lo = quat_rotate(inv_rotation, origin - s.center) * unscale;
    V3 ld = quat_rotate(inv_rotation, heading) * unscale;
    float local_extent = extent * length(ld);
    ShapeHit local;
    if (s.kind == DYN_SHAPE_SPHERE) {
        local = ray_sphere(lo, ld, local_extent, splat3(0.0f), s.radius);
    } else if (s.kind == DYN_SHAPE_CAPSULE) {
        local = ray_capsule(lo, ld, local_extent, splat3(0.0f), V3{0.0f, 1.0f, 0.0f}, s.half_height, s.radius);
    } else if (s.kind == DYN_SHAPE_CYLINDER) {
        local = ray_cylinder(lo, ld, local_extent, splat3(0.0f), V3{0.0f, 1.0f, 0.0f}, s.half_height, s.radius);
    } else {
        return q_no_hit();
    }
    if (local.distance == kNoHit) return q_no_hit();
    ShapeHit hit;
    hit.distance = local.distance;
    hit.triangle = DYN_NO_TRIANGLE;
    hit.point = s.center + quat_rotate(s.rotation, (lo + ld * local.distance) * s.scale);
    hit.normal = quat_rotate(s.rotation, sign_normalize(local.normal * unscale));
    return hit;
}

inline V3 q_origin(const dyn_query_record& q) { return V3{q.origin[0], q.origin[1], q.origin[2]}; }
inline V3 q_direction(const dyn_query_record& q) { return V3{q.direction[0], q.direction[1], q.direction[2]}; }

inline WorldShape query_shape(const dyn_query_record& q, V3 center) {
    WorldShape s;
    s.kind = q.shape_kind;
    s.radius = q.radius;
    s.half_height = q.half_height;
    s.center = center;
    s.half_extents = V3{q.half_extents[0], q.half_extents[1], q.half_extents[2]};
    s.rotation = V4{q.orientation[0], q.orientation[1], q.orientation[2], q.orientation[3]};
    s.source = q.source;
    s.scale = splat3(1.0f);
    return s;
}

// the library's query_probe: a zero orientation (sphere, point and cuboid queries) makes the probe
// its centre point, which is what the reference's zero quaternion does to every support offset
inline WorldShape query_probe(const dyn_query_record& q, V3 center) {
    WorldShape s = query_shape(q, center);
    if (s.rotation.x == 0.0f && s.rotation.y == 0.0f && s.rotation.z == 0.0f && s.rotation.w == 0.0f) {
        s.kind = DYN_SHAPE_SPHERE;
        s.radius = 0.0f;
        s.rotation = V4{0.0f, 0.0f, 0.0f, 1.0f};
    }
    return s;
}

inline ShapeHit penetration_hit(const Shapes& sh, const WorldShape& probe, const WorldShape& solid) {
    ShapeHit h = convex_hit(sh, probe, solid);
    h.normal = -h.normal;
    return h;
}

// overlap_world_geom: the plane's separation, or for another collider only the normal it leaves
// behind (see the library's query.cuh): (0, 1, 0), or the closest hull triangle's (the first
// penetrating one stops the walk)
inline float overlap_world_geom(const Shapes& sh, const HullTriangles& ht, const dyn_query_record& q,
                                const WorldShape& scene, V3* out_normal) {
    if (scene.kind == DYN_SHAPE_PLANE) {
        V3 n = shape_axis(scene);
        *out_normal = n;
        return dot(q_origin(q) - scene.center, n) - q.extent;
    }
    V3 normal = V3{0.0f, 1.0f, 0.0f};
    float distance = kNoHit;
    if (shape_source(scene.kind)) {
        V4 qc = quat_conjugate(scene.rotation);
        WorldShape local = query_probe(q, quat_rotate(qc, q_origin(q) - scene.center));
        local.rotation = quat_mul(qc, local.rotation);
        const dyn_shape_source_record& src = sh.sources[scene.source];
        uint32_t first = ht.ranges[2 * scene.source], count = ht.ranges[2 * scene.source + 1];
        bool found = false;
        for (uint32_t t = 0; t < count; ++t) {
            const uint32_t* tri = ht.tris + 3 * (size_t)(first + t);
            V3 a = hull_corner(sh, src, tri[0], scene.scale), b = hull_corner(sh, src, tri[1], scene.scale),
               c = hull_corner(sh, src, tri[2], scene.scale);
            V3 n = sign_normalize(cross(b - a, c - a));
            float offset = dot(local.center - a, n);
            if (offset < 0.0f) {
                n = -n;
                offset = -offset;
            }
            V3 deep = support(sh, local, -n);
            float extent = dot(deep - local.center, -n);
            float separation = offset - extent;
            bool penetrating = separation < 0.0f;
            if (penetrating || separation < distance) {
                distance = separation;
                normal = n;
                found = true;
                if (penetrating) break;
            }
        }
        if (found) normal = sign_normalize(quat_rotate(scene.rotation, normal));
    }
    *out_normal = normal;
    return distance;
}

inline float overlap_hit(const Shapes& sh, const dyn_query_record& q, const WorldShape& world, V3* out_normal) {
    WorldShape probe = query_probe(q, q_origin(q));
    probe.radius = 0.0f;
    SimplexPoint simplex[4];
    uint32_t count = 0;
    ConvexClosest closest = convex_closest(sh, probe, world, simplex, &count);
    if (closest.penetrating) {
        ShapeHit hit = penetration_hit(sh, query_probe(q, q_origin(q)), world);
        *out_normal = hit.normal;
        return -q.extent + fmaxw(hit.distance + q.extent, 0.0f);
    }
    if (closest.distance <= q.extent) {
        *out_normal = -closest.normal;
        return closest.distance - q.extent;
    }
    return kNoHit;
}

inline ShapeHit shape_sweep(const Shapes& sh, const WorldShape& moving, const WorldShape& target, V3 start, V3 direction,
                            float max_dist) {
    V3 heading = normalize(direction);
    if (target.kind == DYN_SHAPE_PLANE) {
        V3 normal = shape_axis(target);
        float travel = dot(heading, normal);
        if (travel >= 0.0f) return q_no_hit();
        float extent = dot(support(sh, moving, -normal) - moving.center, -normal);
        float offset = dot(start - target.center, normal);
        float time = fmaxw((offset - extent) / (-travel), 0.0f);
        if (time > max_dist) return q_no_hit();
        return ShapeHit{time, start + heading * time, normal, DYN_NO_TRIANGLE};
    }
    WorldShape moved = moving;
    float time = 0.0f;
    V3 normal = sign_normalize(moving.center - target.center);
    for (uint32_t iteration = 0; iteration < 8u; ++iteration) {
        moved.center = start + heading * time;
        SimplexPoint simplex[4];
        uint32_t count = 0;
        ConvexClosest closest = convex_closest(sh, moved, target, simplex, &count);
        if (closest.penetrating || closest.distance < 1e-4f) return ShapeHit{time, start + heading * time, normal, DYN_NO_TRIANGLE};
        normal = -closest.normal;
        time = time + closest.distance;
        if (time > max_dist) return q_no_hit();
    }
    return q_no_hit();
}

inline ShapeHit resolve_hit(const Shapes& sh, const HullTriangles& ht, const dyn_query_record& q, const WorldShape& world) {
    if (q.kind == DYN_QUERY_RAY) {
        V3 direction = normalize(q_direction(q));
        ShapeHit hit = shape_ray(sh, ht, world, q_origin(q), direction, q.extent);
        if (hit.distance == kNoHit) return hit;
        if (dot(hit.normal, direction) > 0.0f) hit.normal = -hit.normal;
        return hit;
    }
    bool world_geom = shape_world_geometry(world.kind);
    if (q.kind == DYN_QUERY_SWEEP) {
        ShapeHit hit = shape_sweep(sh, query_probe(q, q_origin(q)), world, q_origin(q), q_direction(q), q.extent);
        return hit.distance < kNoHit ? hit : q_no_hit();
    }
    V3 normal = splat3(0.0f);
    if (q.kind == DYN_QUERY_SPHERE || q.kind == DYN_QUERY_POINT) {
        float from_hit = overlap_hit(sh, q, world, &normal);
        float from_geom = overlap_world_geom(sh, ht, q, world, &normal);
        float separation = world_geom ? from_geom : from_hit;
        if (separation < kNoHit) return ShapeHit{separation, world.center, normal, DYN_NO_TRIANGLE};
        return q_no_hit();
    }
    if (world_geom) {
        float separation = overlap_world_geom(sh, ht, q, world, &normal);
        if (separation < kNoHit) return ShapeHit{separation, world.center, normal, DYN_NO_TRIANGLE};
        return q_no_hit();
    }
    WorldShape probe = query_probe(q, q_origin(q));
    SimplexPoint simplex[4];
    uint32_t count = 0;
    ConvexClosest closest = convex_closest(sh, probe, world, simplex, &count);
    if (closest.penetrating) {
        ShapeHit hit = penetration_hit(sh, probe, world);
        return ShapeHit{hit.distance, (closest.point_a + closest.point_b) * 0.5f, hit.normal, DYN_NO_TRIANGLE};
    }
    return q_no_hit();
}

inline uint32_t hit_key(float distance) {
    uint32_t bits = f2u(distance);
    return (bits & 0x80000000u) != 0u ? ~bits : (bits | 0x80000000u);
}

}  // namespace orc
