// oracle_geom.h - CPU restatement of the Dynamis narrowphase (contact manifolds).
//
// TEST INFRASTRUCTURE ONLY: part of the oracle that tests/ and bench.py's cpu_baseline leg use as
// the checker. It restates, function by function and in the same operand order:
//   crates/dynamis-shader/shaders/core.wgsl      (bodies, shapes, manifolds)
//   crates/dynamis-shader/shaders/convex.wgsl    (support maps, GJK, EPA, probe, feature clipping)
//   crates/dynamis-rigid/shaders/narrowphase.wgsl (pair filters and the analytic pair kernels)
// Each function cites the WGSL lines it follows. World geometry other than planes (meshes,
// heightfields) and hulls above 4,096 vertices (BVH support) are not restated.
#pragma once

#include <vector>

#include "dynamis_abi.h"
#include "oracle_math.h"

namespace orc {

// ---- loaded records ----

inline V3 rd3(const float* p) { return V3{p[0], p[1], p[2]}; }
inline V4 rd4(const float* p) { return V4{p[0], p[1], p[2], p[3]}; }
inline void wr3(float* p, V3 v) {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}
inline void wr4(float* p, V4 v) {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
    p[3] = v.w;
}

// core.wgsl:1-4 (Body = state + descriptor); only the fields the step reads.
struct Body {
    V3 position;
    V4 orientation;
    V3 velocity;
    V3 angular_velocity;
    uint32_t sleeping;
    uint32_t body_id;
    uint32_t generation;
    float inverse_mass;
    uint32_t flags;
    uint32_t group;
    uint32_t mask;
    V3 com;
    float inverse_inertia[6];
};

inline Body load_body(const dyn_body_state_record& s, const dyn_body_descriptor_record& d) {
    Body b;
    b.position = rd3(s.position);
    b.orientation = rd4(s.orientation);
    b.velocity = rd3(s.velocity);
    b.angular_velocity = rd3(s.angular_velocity);
    b.sleeping = s.sleeping;
    b.body_id = s.body_id;
    b.generation = s.generation;
    b.inverse_mass = d.inverse_mass;
    b.flags = d.flags;
    b.group = d.collision_group;
    b.mask = d.collision_mask;
    b.com = rd3(d.com);
    for (int i = 0; i < 6; ++i) b.inverse_inertia[i] = d.inverse_inertia[i];
    return b;
}

// core.wgsl:188-231 and dynamis-model BodyKind (Dynamic simulates; Static does not move).
inline bool desc_kinematic(uint32_t flags) { return (flags & DYN_BODY_KINEMATIC) != 0u; }
inline bool body_simulates_d(float inverse_mass, uint32_t flags) {
    return !desc_kinematic(flags) && inverse_mass > 0.0f;
}
inline bool body_moves_d(float inverse_mass, uint32_t flags) {
    return desc_kinematic(flags) || inverse_mass > 0.0f;
}
inline bool body_simulates(const Body& b) { return body_simulates_d(b.inverse_mass, b.flags); }
inline bool body_moves(const Body& b) { return body_moves_d(b.inverse_mass, b.flags); }
inline bool body_is_inert(const Body& b) { return !body_simulates(b) || b.sleeping != 0u; }
inline bool body_has_ccd(const Body& b) { return (b.flags & DYN_BODY_CCD) != 0u; }
inline Body body_frozen(Body b) {
    b.inverse_mass = 0.0f;
    for (int i = 0; i < 6; ++i) b.inverse_inertia[i] = 0.0f;
    return b;
}

// core.wgsl:347-394
inline V3 body_com(const Body& b) { return b.position + quat_rotate(b.orientation, b.com); }
inline V3 symmetric_apply(const float* t, V3 v) {
    return V3{t[0] * v.x + t[1] * v.y + t[2] * v.z, t[1] * v.x + t[3] * v.y + t[4] * v.z,
              t[2] * v.x + t[4] * v.y + t[5] * v.z};
}
inline V3 apply_inverse_inertia_of(const float* inverse_inertia, V4 q, V3 v) {
    V3 local = quat_rotate(quat_conjugate(q), v);
    return quat_rotate(q, symmetric_apply(inverse_inertia, local));
}
inline V3 apply_inverse_inertia(const Body& b, V3 v) {
    return apply_inverse_inertia_of(b.inverse_inertia, b.orientation, v);
}
inline V3 point_velocity(const Body& b, V3 point) {
    return b.velocity + cross(b.angular_velocity, point - body_com(b));
}
inline V3 relative_velocity(const Body& a, const Body& b, V3 pa, V3 pb) {
    return point_velocity(b, pb) - point_velocity(a, pa);
}

// ---- shapes ----

struct Shapes {
    const dyn_shape_source_record* sources = nullptr;
    uint32_t source_count = 0;
    const V4* vertices = nullptr;
    uint32_t vertex_count = 0;
};

// core.wgsl:34-43
struct WorldShape {
    uint32_t kind;
    float radius;
    float half_height;
    V3 center;
    V3 half_extents;
    V4 rotation;
    uint32_t source;
    V3 scale;
};

// core.wgsl:473-484
inline WorldShape world_collider(V3 position, V4 orientation, const dyn_collider_record& c) {
    WorldShape w;
    w.kind = c.kind;
    w.radius = c.radius;
    w.half_height = c.half_height;
    w.center = position + quat_rotate(orientation, rd3(c.local_offset));
    w.half_extents = rd3(c.half_extents);
    w.rotation = quat_mul(orientation, rd4(c.local_rotation));
    w.source = c.source;
    w.scale = rd3(c.scale);
    return w;
}

inline bool shape_world_geometry(uint32_t kind) {
    return kind == DYN_SHAPE_MESH || kind == DYN_SHAPE_HEIGHTFIELD || kind == DYN_SHAPE_PLANE;
}
inline bool shape_analytic(uint32_t kind) {
    return kind == DYN_SHAPE_SPHERE || kind == DYN_SHAPE_CUBOID || kind == DYN_SHAPE_CAPSULE;
}
inline bool shape_source(uint32_t kind) {
    return kind == DYN_SHAPE_HULL || kind == DYN_SHAPE_MESH || kind == DYN_SHAPE_HEIGHTFIELD
        || kind == DYN_SHAPE_TRIANGLE;
}

inline V3 shape_axis(const WorldShape& w) { return quat_rotate(w.rotation, V3{0.0f, 1.0f, 0.0f}); }

struct Aabb {
    V3 min, max;
};

// core.wgsl:490-503
inline Aabb world_shape_bounds(const Shapes& sh, const WorldShape& w) {
    const dyn_shape_source_record& src = sh.sources[w.source];
    V3 scaled_min = rd3(src.local_min) * w.scale;
    V3 scaled_max = rd3(src.local_max) * w.scale;
    V3 center = w.center + quat_rotate(w.rotation, (scaled_min + scaled_max) * 0.5f);
    V3 half = (scaled_max - scaled_min) * 0.5f;
    V3 extent = vabs(quat_rotate(w.rotation, V3{half.x, 0.0f, 0.0f}))
        + vabs(quat_rotate(w.rotation, V3{0.0f, half.y, 0.0f}))
        + vabs(quat_rotate(w.rotation, V3{0.0f, 0.0f, half.z}));
    return Aabb{center - extent, center + extent};
}

// core.wgsl:505-536
inline Aabb world_aabb_of(const Shapes& sh, const WorldShape& w) {
    if (w.kind == DYN_SHAPE_PLANE) {
        return Aabb{w.center - splat3(1e6f), w.center + splat3(1e6f)};
    }
    if (shape_source(w.kind)) {
        return world_shape_bounds(sh, w);
    }
    V3 extent = splat3(0.0f);
    if (w.kind == DYN_SHAPE_SPHERE) {
        extent = splat3(w.radius);
    } else if (w.kind == DYN_SHAPE_CUBOID) {
        V3 e = w.half_extents;
        extent = vabs(quat_rotate(w.rotation, V3{e.x, 0.0f, 0.0f}))
            + vabs(quat_rotate(w.rotation, V3{0.0f, e.y, 0.0f}))
            + vabs(quat_rotate(w.rotation, V3{0.0f, 0.0f, e.z}));
    } else if (w.kind == DYN_SHAPE_CAPSULE || w.kind == DYN_SHAPE_CYLINDER) {
        V3 axis = shape_axis(w);
        extent = vabs(axis * w.half_height) + splat3(w.radius);
    }
    float s = fmaxw(fmaxw(w.scale.x, w.scale.y), w.scale.z);
    extent = extent * s;
    return Aabb{w.center - extent, w.center + extent};
}

// ---- manifolds: core.wgsl:614-760 ----

constexpr uint32_t kFeatureMax = 8;
constexpr float kClipMargin = 1e-4f;
constexpr uint32_t kManifoldCandidates = 16;

inline uint32_t feature_pair(uint32_t kind, uint32_t first, uint32_t second) {
    return kind | (first << DYN_FEATURE_FIELD_BITS) | second;
}
inline uint32_t feature_vertex(uint32_t f, uint32_t s) { return feature_pair(DYN_FEATURE_VERTEX, f, s); }
inline uint32_t feature_edge(uint32_t f, uint32_t s) { return feature_pair(DYN_FEATURE_EDGE, f, s); }
inline uint32_t feature_face(uint32_t f, uint32_t s) { return feature_pair(DYN_FEATURE_FACE, f, s); }
inline uint32_t feature_field_clip(uint32_t id) { return DYN_FEATURE_CLIP | id; }
inline uint32_t feature_field_face(uint32_t id) { return DYN_FEATURE_FACE_BIT | id; }
inline uint32_t feature_mirror(uint32_t feature) {
    uint32_t kind = feature & DYN_FEATURE_KIND_MASK;
    if (kind == DYN_FEATURE_POINT) return feature;
    uint32_t first = (feature >> DYN_FEATURE_FIELD_BITS) & DYN_FEATURE_FIELD_MASK;
    uint32_t second = feature & DYN_FEATURE_FIELD_MASK;
    return kind | (second << DYN_FEATURE_FIELD_BITS) | first;
}

struct Candidate {
    V3 position;
    float depth;
    uint32_t feature;
};

// The per-pair contact a kernel builds before material and anchors (Contact fields it touches).
struct Manifold {
    uint32_t point_count = 0;
    V3 normal{0.0f, 0.0f, 0.0f};
    uint32_t triangle = DYN_NO_TRIANGLE;
    Candidate points[DYN_CONTACT_MAX_POINTS];
};

inline void manifold_emit(Manifold* m, V3 normal) {
    m->point_count = 0;
    m->normal = normal;
    m->triangle = DYN_NO_TRIANGLE;
}
inline void manifold_push(Manifold* m, V3 point, float depth, uint32_t feature) {
    if (m->point_count >= DYN_CONTACT_MAX_POINTS) return;
    m->points[m->point_count] = Candidate{point, depth, feature};
    m->point_count += 1;
}
inline void mirror_features(Manifold* m) {
    for (uint32_t i = 0; i < m->point_count; ++i) m->points[i].feature = feature_mirror(m->points[i].feature);
}
inline float manifold_gap(const Candidate* c, uint32_t kept, uint32_t index) {
    float gap = 3.402823466e38f;
    for (uint32_t held = 0; held < kept; ++held) {
        gap = fminw(gap, length(c[index].position - c[held].position));
    }
    return gap;
}
inline void manifold_order(Candidate* c, uint32_t count) {
    uint32_t lead = 0;
    for (uint32_t i = 1; i < count; ++i) {
        float depth = c[i].depth;
        float held = c[lead].depth;
        if (depth > held || (depth == held && c[i].feature < c[lead].feature)) lead = i;
    }
    std::swap(c[0], c[lead]);
    for (uint32_t kept = 1; kept < count; ++kept) {
        uint32_t best = kept;
        float best_gap = manifold_gap(c, kept, kept);
        for (uint32_t i = kept + 1; i < count; ++i) {
            float gap = manifold_gap(c, kept, i);
            if (gap > best_gap) {
                best_gap = gap;
                best = i;
            }
        }
        if (best != kept) std::swap(c[kept], c[best]);
    }
}
inline uint32_t manifold_keep(Manifold* m, Candidate* c, uint32_t count) {
    manifold_order(c, count);
    for (uint32_t i = 0; i < count && m->point_count < DYN_CONTACT_MAX_POINTS; ++i) {
        manifold_push(m, c[i].position, c[i].depth, c[i].feature);
    }
    return m->point_count;
}

// ---- analytic pairs: narrowphase.wgsl:33-473 ----

inline V3 box_center(V3 position, V4 orientation, const dyn_collider_record& c) {
    return position + quat_rotate(orientation, rd3(c.local_offset));
}
inline void box_rotated_axes(V4 orientation, const dyn_collider_record& c, V3 axes[3]) {
    V4 q = quat_mul(orientation, rd4(c.local_rotation));
    axes[0] = quat_rotate(q, V3{1.0f, 0.0f, 0.0f});
    axes[1] = quat_rotate(q, V3{0.0f, 1.0f, 0.0f});
    axes[2] = quat_rotate(q, V3{0.0f, 0.0f, 1.0f});
}
// core.wgsl:586-612
inline V3 closest_point_box(V3 point, const Body& b, const dyn_collider_record& c) {
    V4 q = quat_mul(b.orientation, rd4(c.local_rotation));
    V3 center = box_center(b.position, b.orientation, c);
    V3 local = quat_rotate(quat_conjugate(q), point - center);
    V3 he = rd3(c.half_extents);
    V3 clamped = vclamp(local, -he, he);
    return box_center(b.position, b.orientation, c) + quat_rotate(q, clamped);
}
inline V3 closest_point_segment(V3 point, V3 a, V3 b) {
    V3 ab = b - a;
    float denom = dot(ab, ab);
    if (denom < 1e-10f) return a;
    float t = clampw(dot(point - a, ab) / denom, 0.0f, 1.0f);
    return a + ab * t;
}
inline uint32_t smallest_axis(V3 v) {
    V3 av = vabs(v);
    if (av.x < av.y && av.x < av.z) return 0;
    if (av.y < av.z) return 1;
    return 2;
}

// narrowphase.wgsl:33-57
inline Manifold sphere_sphere(const Body& first, const dyn_collider_record& fc, const Body& second,
                              const dyn_collider_record& sc, float margin) {
    Manifold m;
    V3 first_center = box_center(first.position, first.orientation, fc);
    V3 second_center = box_center(second.position, second.orientation, sc);
    V3 delta = second_center - first_center;
    float distance = length(delta);
    V3 normal = sign_normalize(delta);
    if (distance <= 1e-6f) {
        V3 rel = relative_velocity(first, second, second_center, first_center);
        if (length(rel) > 1e-6f) normal = -normalize(rel);
    }
    manifold_emit(&m, normal);
    float radius_sum = fc.radius + sc.radius;
    if (distance > radius_sum + margin) return m;
    float depth = radius_sum - distance;
    V3 point = first_center + normal * (fc.radius - depth * 0.5f);
    manifold_push(&m, point, depth, DYN_FEATURE_POINT);
    return m;
}

struct BoxFace {
    V3 normal;
    float clearance;
    uint32_t index;
};
// narrowphase.wgsl:65-83
inline BoxFace box_nearest_face(V3 point, const Body& b, const dyn_collider_record& c) {
    V4 q = quat_mul(b.orientation, rd4(c.local_rotation));
    V3 local = quat_rotate(quat_conjugate(q), point - box_center(b.position, b.orientation, c));
    V3 clearance = rd3(c.half_extents) - vabs(local);
    uint32_t axis = smallest_axis(clearance);
    V3 facing = splat3(0.0f);
    if (axis == 0) {
        facing = V3{local.x > 0.0f ? -1.0f : 1.0f, 0.0f, 0.0f};
    } else if (axis == 1) {
        facing = V3{0.0f, local.y > 0.0f ? -1.0f : 1.0f, 0.0f};
    } else {
        facing = V3{0.0f, 0.0f, local.z > 0.0f ? -1.0f : 1.0f};
    }
    BoxFace face;
    face.normal = -quat_rotate(q, facing);
    face.clearance = comp(clearance, axis);
    face.index = axis * 2u + (comp(local, axis) > 0.0f ? 1u : 0u);
    return face;
}
// narrowphase.wgsl:85-110
inline Manifold sphere_box(const Body& sphere, const dyn_collider_record& scol, const Body& box,
                           const dyn_collider_record& bcol, float margin) {
    Manifold m;
    V3 center = sphere.position + quat_rotate(sphere.orientation, rd3(scol.local_offset));
    V3 closest = closest_point_box(center, box, bcol);
    V3 delta = closest - center;
    float distance = length(delta);
    float radius = scol.radius;
    V3 normal = sign_normalize(delta);
    float depth = radius - distance;
    if (distance <= 1e-6f) {
        BoxFace face = box_nearest_face(center, box, bcol);
        normal = -face.normal;
        depth = radius + face.clearance;
    }
    manifold_emit(&m, normal);
    if (depth <= -margin) return m;
    V3 point = closest - normal * (depth * 0.5f);
    manifold_push(&m, point, depth, DYN_FEATURE_POINT);
    return m;
}
struct Segment {
    V3 start, end;
};
// narrowphase.wgsl:112-117
inline Segment capsule_segment(const Body& b, const dyn_collider_record& c) {
    V4 q = quat_mul(b.orientation, rd4(c.local_rotation));
    V3 axis = quat_rotate(q, V3{0.0f, 1.0f, 0.0f});
    V3 center = box_center(b.position, b.orientation, c);
    return Segment{center - axis * c.half_height, center + axis * c.half_height};
}
// narrowphase.wgsl:119-140
inline Manifold sphere_capsule(const Body& sphere, const dyn_collider_record& scol, const Body& cap,
                               const dyn_collider_record& ccol, float margin) {
    Manifold m;
    Segment seg = capsule_segment(cap, ccol);
    V3 center = sphere.position + quat_rotate(sphere.orientation, rd3(scol.local_offset));
    V3 closest = closest_point_segment(center, seg.start, seg.end);
    V3 delta = closest - center;
    float distance = length(delta);
    float radius_sum = scol.radius + ccol.radius;
    manifold_emit(&m, sign_normalize(delta));
    if (distance > radius_sum + margin) return m;
    V3 normal = sign_normalize(delta);
    float depth = radius_sum - distance;
    V3 point = closest - normal * (depth * 0.5f);
    manifold_push(&m, point, depth, DYN_FEATURE_POINT);
    return m;
}
// narrowphase.wgsl:142-181
inline Segment closest_points_segments(V3 a0, V3 a1, V3 b0, V3 b1) {
    V3 d1 = a1 - a0;
    V3 d2 = b1 - b0;
    V3 r = a0 - b0;
    float a = dot(d1, d1);
    float e = dot(d2, d2);
    float f = dot(d2, r);
    float s = 0.0f;
    float t = 0.0f;
    if (a <= 1e-10f && e <= 1e-10f) {
        s = 0.0f;
        t = 0.0f;
    } else if (a <= 1e-10f) {
        s = 0.0f;
        t = clampw(f / e, 0.0f, 1.0f);
    } else {
        float c = dot(d1, r);
        if (e <= 1e-10f) {
            t = 0.0f;
            s = clampw(-c / a, 0.0f, 1.0f);
        } else {
            float b = dot(d1, d2);
            float denom = a * e - b * b;
            if (denom != 0.0f) {
                s = clampw((b * f - c * e) / denom, 0.0f, 1.0f);
            } else {
                s = 0.0f;
            }
            t = (b * s + f) / e;
            if (t < 0.0f) {
                t = 0.0f;
                s = clampw(-c / a, 0.0f, 1.0f);
            } else if (t > 1.0f) {
                t = 1.0f;
                s = clampw((b - c) / a, 0.0f, 1.0f);
            }
        }
    }
    return Segment{a0 + d1 * s, b0 + d2 * t};
}
// narrowphase.wgsl:183-204
inline Manifold capsule_capsule(const Body& first, const dyn_collider_record& fc, const Body& second,
                                const dyn_collider_record& sc, float margin) {
    Manifold m;
    Segment a = capsule_segment(first, fc);
    Segment b = capsule_segment(second, sc);
    Segment closest = closest_points_segments(a.start, a.end, b.start, b.end);
    V3 delta = closest.end - closest.start;
    float distance = length(delta);
    float radius_sum = fc.radius + sc.radius;
    manifold_emit(&m, sign_normalize(delta));
    if (distance > radius_sum + margin) return m;
    float depth = radius_sum - distance;
    V3 point = (closest.start + closest.end) * 0.5f;
    manifold_push(&m, point, depth, DYN_FEATURE_POINT);
    return m;
}

// convex.wgsl:625-631
inline uint32_t box_corner_id(uint32_t face_axis, float face_sign, float first, float second) {
    uint32_t id = 0;
    id |= face_sign > 0.0f ? (1u << face_axis) : 0u;
    id |= first > 0.0f ? (1u << ((face_axis + 1u) % 3u)) : 0u;
    id |= second > 0.0f ? (1u << ((face_axis + 2u) % 3u)) : 0u;
    return id;
}

// narrowphase.wgsl:206-213
inline V3 box_support(const Body& b, const dyn_collider_record& c, V3 direction) {
    V3 axes[3];
    box_rotated_axes(b.orientation, c, axes);
    V3 point = box_center(b.position, b.orientation, c);
    for (uint32_t i = 0; i < 3; ++i) {
        float h = comp(rd3(c.half_extents), i);
        point = point + axes[i] * (dot(axes[i], direction) > 0.0f ? h : -h);
    }
    return point;
}
// narrowphase.wgsl:215-252
inline V3 box_face(const Body& b, const dyn_collider_record& c, V3 face_normal, V3 corners[4],
                   uint32_t ids[4], uint32_t* out_face) {
    V3 axes[3];
    box_rotated_axes(b.orientation, c, axes);
    V3 center = box_center(b.position, b.orientation, c);
    V3 he = rd3(c.half_extents);
    uint32_t axis = 0;
    for (uint32_t i = 1; i < 3; ++i) {
        if (std::fabs(dot(face_normal, axes[i])) > std::fabs(dot(face_normal, axes[axis]))) axis = i;
    }
    float sign = dot(face_normal, axes[axis]) < 0.0f ? -1.0f : 1.0f;
    V3 n = axes[axis] * sign;
    V3 u = axes[(axis + 1u) % 3u];
    V3 v = axes[(axis + 2u) % 3u];
    float half_u = comp(he, (axis + 1u) % 3u);
    float half_v = comp(he, (axis + 2u) % 3u);
    V3 face_center = center + n * comp(he, axis);
    V3 edges[4];
    edges[0] = u * half_u + v * half_v;
    edges[1] = -u * half_u + v * half_v;
    edges[2] = -u * half_u - v * half_v;
    edges[3] = u * half_u - v * half_v;
    for (uint32_t i = 0; i < 4; ++i) corners[i] = face_center + edges[i];
    ids[0] = box_corner_id(axis, sign, 1.0f, 1.0f);
    ids[1] = box_corner_id(axis, sign, -1.0f, 1.0f);
    ids[2] = box_corner_id(axis, sign, -1.0f, -1.0f);
    ids[3] = box_corner_id(axis, sign, 1.0f, -1.0f);
    *out_face = axis * 2u + (sign > 0.0f ? 1u : 0u);
    return face_center;
}
// narrowphase.wgsl:254-288
inline uint32_t clip_polygon(const V3* points, const uint32_t* ids, uint32_t count, V3 plane_point,
                             V3 plane_normal, uint32_t group, uint32_t side, V3* out_points,
                             uint32_t* out_ids) {
    uint32_t out_count = 0;
    for (uint32_t i = 0; i < count; ++i) {
        V3 current = points[i];
        V3 next = points[(i + 1u) % count];
        float current_dist = dot(current - plane_point, plane_normal) - kClipMargin;
        float next_dist = dot(next - plane_point, plane_normal) - kClipMargin;
        if (current_dist <= 0.0f) {
            if (out_count < 8u) {
                out_points[out_count] = current;
                out_ids[out_count] = ids[i];
                out_count += 1;
            }
        }
        if (current_dist * next_dist < 0.0f) {
            float t = current_dist / (current_dist - next_dist);
            if (out_count < 8u) {
                out_points[out_count] = current + (next - current) * t;
                out_ids[out_count] = feature_field_clip(group * 32u + side * 8u + i);
                out_count += 1;
            }
        }
    }
    return out_count;
}

constexpr float kFaceAxisBias = 1e-3f;

struct BoxGeometry {
    const Body* body;
    const dyn_collider_record* collider;
    V3 axes[3];
    V3 half_extents;
    V3 center;
};
inline BoxGeometry box_geometry(const Body& b, const dyn_collider_record& c) {
    BoxGeometry g;
    g.body = &b;
    g.collider = &c;
    box_rotated_axes(b.orientation, c, g.axes);
    g.half_extents = rd3(c.half_extents);
    g.center = box_center(b.position, b.orientation, c);
    return g;
}
inline float support_radius(const BoxGeometry& g, V3 axis) {
    return std::fabs(dot(g.axes[0], axis)) * g.half_extents.x
        + std::fabs(dot(g.axes[1], axis)) * g.half_extents.y
        + std::fabs(dot(g.axes[2], axis)) * g.half_extents.z;
}
inline float face_overlap(const BoxGeometry& face, const BoxGeometry& other, uint32_t axis_index, V3 delta) {
    V3 axis = face.axes[axis_index];
    return comp(face.half_extents, axis_index) + support_radius(other, axis) - std::fabs(dot(delta, axis));
}
inline float edge_overlap(const BoxGeometry& l, const BoxGeometry& r, V3 axis, V3 delta) {
    return support_radius(l, axis) + support_radius(r, axis) - std::fabs(dot(delta, axis));
}

// narrowphase.wgsl:325-473
inline Manifold box_box_sat(const Body& first, const dyn_collider_record& fc, const Body& second,
                            const dyn_collider_record& sc, float margin) {
    Manifold m;
    BoxGeometry left = box_geometry(first, fc);
    BoxGeometry right = box_geometry(second, sc);
    V3 delta = right.center - left.center;
    float face_depth = 1e30f;
    V3 face_axis = left.axes[0];
    bool face_on_right = false;
    for (uint32_t i = 0; i < 3; ++i) {
        float overlap = face_overlap(left, right, i, delta);
        if (overlap < face_depth) {
            face_depth = overlap;
            face_axis = left.axes[i];
            face_on_right = false;
        }
        float other = face_overlap(right, left, i, delta);
        if (other < face_depth) {
            face_depth = other;
            face_axis = right.axes[i];
            face_on_right = true;
        }
    }
    float edge_depth = 1e30f;
    V3 edge_axis = face_axis;
    uint32_t edge_first_axis = 0, edge_second_axis = 0;
    for (uint32_t i = 0; i < 3; ++i) {
        for (uint32_t j = 0; j < 3; ++j) {
            V3 crossed = cross(left.axes[i], right.axes[j]);
            float len = length(crossed);
            if (len < 1e-8f) continue;
            V3 axis = crossed / len;
            float overlap = edge_overlap(left, right, axis, delta);
            if (overlap < edge_depth) {
                edge_depth = overlap;
                edge_axis = axis;
                edge_first_axis = i;
                edge_second_axis = j;
            }
        }
    }
    float extent = fmaxw(fmaxw(left.half_extents.x, left.half_extents.y), left.half_extents.z)
        + fmaxw(fmaxw(right.half_extents.x, right.half_extents.y), right.half_extents.z);
    bool edge_axis_separates = edge_depth + kFaceAxisBias * extent < face_depth;
    float depth = edge_axis_separates ? edge_depth : face_depth;
    if (depth <= -margin) return m;
    V3 axis = edge_axis_separates ? edge_axis : face_axis;
    V3 signed_axis = dot(axis, delta) < 0.0f ? -axis : axis;
    manifold_emit(&m, signed_axis);
    if (edge_axis_separates) {
        V3 point = (box_support(first, fc, signed_axis) + box_support(second, sc, -signed_axis)) * 0.5f;
        manifold_push(&m, point, depth, feature_edge(edge_first_axis, edge_second_axis));
        return m;
    }
    const BoxGeometry* reference = &left;
    const BoxGeometry* incident = &right;
    V3 ref_normal = signed_axis;
    if (face_on_right) {
        reference = &right;
        incident = &left;
        ref_normal = -signed_axis;
    }
    V3 ref_corners[4];
    uint32_t ref_ids[4];
    uint32_t ref_face = 0;
    V3 ref_center = box_face(*reference->body, *reference->collider, ref_normal, ref_corners, ref_ids, &ref_face);
    uint32_t incident_axis = 0;
    for (uint32_t i = 1; i < 3; ++i) {
        if (std::fabs(dot(incident->axes[i], ref_normal)) > std::fabs(dot(incident->axes[incident_axis], ref_normal))) {
            incident_axis = i;
        }
    }
    V3 incident_normal = incident->axes[incident_axis]
        * (dot(incident->axes[incident_axis], ref_normal) > 0.0f ? -1.0f : 1.0f);
    V3 incident_corners[4];
    uint32_t incident_ids[4];
    uint32_t incident_face = 0;
    box_face(*incident->body, *incident->collider, incident_normal, incident_corners, incident_ids, &incident_face);
    uint32_t ref_field = feature_field_face(ref_face);
    V3 poly_a[8], poly_b[8];
    uint32_t ids_a[8], ids_b[8];
    for (uint32_t i = 0; i < 4; ++i) {
        poly_a[i] = incident_corners[i];
        ids_a[i] = incident_ids[i];
    }
    uint32_t polygon_count = 4;
    for (uint32_t side = 0; side < 4; ++side) {
        V3 current = ref_corners[side];
        V3 next = ref_corners[(side + 1u) % 4u];
        V3 plane_normal = normalize(cross(next - current, ref_normal));
        if (side % 2u == 0u) {
            polygon_count = clip_polygon(poly_a, ids_a, polygon_count, current, plane_normal, incident_face, side, poly_b, ids_b);
        } else {
            polygon_count = clip_polygon(poly_b, ids_b, polygon_count, current, plane_normal, incident_face, side, poly_a, ids_a);
        }
        if (polygon_count == 0u) break;
    }
    Candidate candidates[kManifoldCandidates];
    uint32_t candidate_count = 0;
    for (uint32_t i = 0; i < polygon_count && candidate_count < kManifoldCandidates; ++i) {
        float point_depth = dot(ref_center - poly_a[i], ref_normal);
        if (point_depth >= -margin) {
            candidates[candidate_count] = Candidate{
                poly_a[i] - ref_normal * (point_depth * 0.5f), point_depth,
                face_on_right ? feature_face(ids_a[i], ref_field) : feature_face(ref_field, ids_a[i])};
            candidate_count += 1;
        }
    }
    if (candidate_count == 0u) {
        for (uint32_t i = 0; i < 4 && candidate_count < kManifoldCandidates; ++i) {
            float point_depth = dot(ref_center - incident_corners[i], ref_normal);
            if (point_depth >= -margin) {
                candidates[candidate_count] = Candidate{
                    incident_corners[i] - ref_normal * (point_depth * 0.5f), point_depth,
                    face_on_right ? feature_face(incident_ids[i], ref_field) : feature_face(ref_field, incident_ids[i])};
                candidate_count += 1;
            }
        }
    }
    if (candidate_count == 0u) {
        manifold_push(&m, ref_center - ref_normal * (face_depth * 0.5f), face_depth, DYN_FEATURE_POINT);
        return m;
    }
    manifold_keep(&m, candidates, candidate_count);
    return m;
}

// ---- convex support maps: convex.wgsl:1-91 ----

constexpr uint32_t kLinearSupportVertices = 4096;

inline V3 support_local(const Shapes& sh, const WorldShape& w, V3 direction) {
    V3 d = direction;
    V3 n = normalize(direction);
    if (w.kind == DYN_SHAPE_SPHERE) return n * w.radius;
    if (w.kind == DYN_SHAPE_CUBOID) {
        V3 signs = V3{d.x > 0.0f ? 1.0f : -1.0f, d.y > 0.0f ? 1.0f : -1.0f, d.z > 0.0f ? 1.0f : -1.0f};
        return signs * w.half_extents;
    }
    if (w.kind == DYN_SHAPE_CAPSULE) {
        V3 tip = V3{0.0f, 1.0f, 0.0f} * w.half_height * (d.y > 0.0f ? 1.0f : -1.0f);
        return tip + n * w.radius;
    }
    if (w.kind == DYN_SHAPE_CYLINDER) {
        V3 base = V3{0.0f, 1.0f, 0.0f} * w.half_height * (d.y > 0.0f ? 1.0f : -1.0f);
        V3 radial = d - V3{0.0f, d.y, 0.0f};
        if (length(radial) < 1e-6f) return base;
        return base + normalize(radial) * w.radius;
    }
    const dyn_shape_source_record& src = sh.sources[w.source];
    float best_dot = -3.402823466e38f;
    V3 best = splat3(0.0f);
    for (uint32_t i = 0; i < src.vertex_count; ++i) {
        V3 v = xyz(sh.vertices[src.vertex_offset + i]);
        float s = dot(v, d);
        if (s > best_dot) {
            best_dot = s;
            best = v;
        }
    }
    return best;
}
inline V3 support(const Shapes& sh, const WorldShape& w, V3 direction) {
    V3 local_d = quat_rotate(quat_conjugate(w.rotation), direction);
    V3 scaled_d = local_d * w.scale;
    V3 local = support_local(sh, w, scaled_d);
    return w.center + quat_rotate(w.rotation, local * w.scale);
}

// ---- GJK: convex.wgsl:93-278, 439-521 ----

struct SimplexPoint {
    V3 w, a, b;
};
struct SimplexResult {
    V3 v;
    float lambdas[4];
    bool penetrating;
    V3 point_a, point_b;
};

inline V3 closest_on_triangle(V3 origin, V3 a, V3 b, V3 c, V3* out_weights) {
    V3 ab = b - a;
    V3 ac = c - a;
    V3 ap = origin - a;
    float d1 = dot(ab, ap);
    float d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) {
        *out_weights = V3{1.0f, 0.0f, 0.0f};
        return a;
    }
    V3 bp = origin - b;
    float d3 = dot(ab, bp);
    float d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) {
        *out_weights = V3{0.0f, 1.0f, 0.0f};
        return b;
    }
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float t = d1 / (d1 - d3);
        *out_weights = V3{1.0f - t, t, 0.0f};
        return a + ab * t;
    }
    V3 cp = origin - c;
    float d5 = dot(ab, cp);
    float d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) {
        *out_weights = V3{0.0f, 0.0f, 1.0f};
        return c;
    }
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        float t = d2 / (d2 - d6);
        *out_weights = V3{1.0f - t, 0.0f, t};
        return a + ac * t;
    }
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        *out_weights = V3{0.0f, 1.0f - t, t};
        return b + (c - b) * t;
    }
    float denom = 1.0f / (va + vb + vc);
    float v = vb * denom;
    float w = vc * denom;
    *out_weights = V3{1.0f - v - w, v, w};
    return a + ab * v + ac * w;
}
inline float face_span(V3 a, V3 b, V3 c) {
    return fmaxw(fmaxw(length(b - a), length(c - a)), length(c - b));
}
inline void tetra_face(const SimplexPoint* tet, uint32_t face, V3* a, V3* b, V3* c) {
    if (face == 0) {
        *a = tet[0].w; *b = tet[1].w; *c = tet[2].w;
    } else if (face == 1) {
        *a = tet[0].w; *b = tet[2].w; *c = tet[3].w;
    } else if (face == 2) {
        *a = tet[0].w; *b = tet[3].w; *c = tet[1].w;
    } else {
        *a = tet[1].w; *b = tet[3].w; *c = tet[2].w;
    }
}
inline bool tetra_contains(const SimplexPoint* tet, V3 origin) {
    for (uint32_t face = 0; face < 4; ++face) {
        V3 a, b, c;
        tetra_face(tet, face, &a, &b, &c);
        V3 normal = cross(b - a, c - a);
        float span = face_span(a, b, c);
        if (length(normal) <= 1e-6f * span * span) return false;
        if (dot(normal, origin - a) > 0.0f) return false;
    }
    return true;
}
inline bool simplex_holds(const SimplexPoint* s, uint32_t count, V3 point, float span) {
    float tolerance = (1e-5f * span) * (1e-5f * span);
    for (uint32_t i = 0; i < count; ++i) {
        V3 offset = s[i].w - point;
        if (dot(offset, offset) <= tolerance) return true;
    }
    return false;
}
inline uint32_t simplex_reduce(SimplexPoint* s, const float* lambdas) {
    SimplexPoint kept[4];
    uint32_t count = 0;
    for (uint32_t i = 0; i < 4; ++i) {
        if (lambdas[i] > 1e-6f) {
            kept[count] = s[i];
            count += 1;
        }
    }
    if (count == 0) {
        kept[0] = s[0];
        count = 1;
    }
    for (uint32_t i = 0; i < count; ++i) s[i] = kept[i];
    return count;
}
inline SimplexResult simplex_closest(const SimplexPoint* s, uint32_t count) {
    SimplexResult r;
    r.v = splat3(3.402823466e38f);
    for (int i = 0; i < 4; ++i) r.lambdas[i] = 0.0f;
    r.penetrating = count == 4u && tetra_contains(s, splat3(0.0f));
    r.point_a = splat3(0.0f);
    r.point_b = splat3(0.0f);
    if (r.penetrating) {
        r.v = splat3(0.0f);
        return r;
    }
    for (uint32_t i = 0; i < count; ++i) {
        float d = length(s[i].w);
        if (d < length(r.v)) {
            r.v = s[i].w;
            for (int k = 0; k < 4; ++k) r.lambdas[k] = 0.0f;
            r.lambdas[i] = 1.0f;
        }
    }
    for (uint32_t i = 0; i < count; ++i) {
        for (uint32_t j = i + 1; j < count; ++j) {
            V3 a = s[i].w;
            V3 b = s[j].w;
            V3 ab = b - a;
            float denom = dot(ab, ab);
            if (denom < 1e-12f) continue;
            float t = clampw(-dot(a, ab) / denom, 0.0f, 1.0f);
            V3 point = a + ab * t;
            if (length(point) < length(r.v)) {
                r.v = point;
                for (int k = 0; k < 4; ++k) r.lambdas[k] = 0.0f;
                r.lambdas[i] = 1.0f - t;
                r.lambdas[j] = t;
            }
        }
    }
    if (count >= 3u) {
        for (uint32_t i = 0; i < count; ++i) {
            for (uint32_t j = i + 1; j < count; ++j) {
                for (uint32_t k = j + 1; k < count; ++k) {
                    V3 weights = splat3(0.0f);
                    V3 point = closest_on_triangle(splat3(0.0f), s[i].w, s[j].w, s[k].w, &weights);
                    if (length(point) < length(r.v)) {
                        r.v = point;
                        for (int q = 0; q < 4; ++q) r.lambdas[q] = 0.0f;
                        r.lambdas[i] = weights.x;
                        r.lambdas[j] = weights.y;
                        r.lambdas[k] = weights.z;
                    }
                }
            }
        }
    }
    for (uint32_t i = 0; i < count; ++i) {
        r.point_a = r.point_a + r.lambdas[i] * s[i].a;
        r.point_b = r.point_b + r.lambdas[i] * s[i].b;
    }
    return r;
}
inline SimplexPoint support_pair(const Shapes& sh, const WorldShape& f, const WorldShape& s, V3 direction) {
    V3 a = support(sh, f, direction);
    V3 b = support(sh, s, -direction);
    return SimplexPoint{a - b, a, b};
}

struct EpaResult {
    bool valid;
    V3 normal;
    float depth;
    V3 point;
};
struct EpaFace {
    uint32_t a, b, c;
    V3 normal;
};

// convex.wgsl:286-437
inline EpaResult epa_tetrahedron(const Shapes& sh, const WorldShape& first, const WorldShape& second,
                                 const SimplexPoint* simplex, uint32_t count) {
    SimplexPoint polytope[64];
    EpaFace new_faces[64];
    EpaFace faces[128];
    uint32_t visible[128];
    uint32_t vertex_count = 0;
    for (uint32_t i = 0; i < count; ++i) {
        polytope[vertex_count] = simplex[i];
        vertex_count += 1;
    }
    uint32_t face_count = 0;
    EpaResult invalid{false, V3{0.0f, 1.0f, 0.0f}, 0.0f, splat3(0.0f)};
    if (vertex_count != 4u) return invalid;
    static const uint32_t kTet[4][3] = {{0, 1, 2}, {0, 2, 3}, {0, 3, 1}, {1, 3, 2}};
    for (uint32_t i = 0; i < 4; ++i) {
        uint32_t a = kTet[i][0], b = kTet[i][1], c = kTet[i][2];
        V3 normal = cross(polytope[b].w - polytope[a].w, polytope[c].w - polytope[a].w);
        float length_n = length(normal);
        if (length_n < 1e-10f) return invalid;
        V3 unit = normal / length_n;
        V3 centroid = (polytope[a].w + polytope[b].w + polytope[c].w) * (1.0f / 3.0f);
        faces[face_count] = EpaFace{a, b, c, dot(unit, centroid) > 0.0f ? -unit : unit};
        face_count += 1;
    }
    float best_dist = 0.0f;
    uint32_t best_face = 0;
    for (uint32_t iter = 0; iter < 32u; ++iter) {
        best_dist = 3.402823466e38f;
        best_face = 0;
        for (uint32_t i = 0; i < face_count; ++i) {
            float dist = dot(faces[i].normal, polytope[faces[i].a].w);
            if (dist < best_dist && length(faces[i].normal) > 0.5f) {
                best_dist = dist;
                best_face = i;
            }
        }
        V3 probe = support_pair(sh, first, second, faces[best_face].normal).w;
        float gain = dot(probe, faces[best_face].normal) - best_dist;
        if (gain < 1e-4f) break;
        if (vertex_count >= 64u) break;
        polytope[vertex_count] = SimplexPoint{probe, support(sh, first, faces[best_face].normal),
                                              support(sh, second, -faces[best_face].normal)};
        vertex_count += 1;
        uint32_t visible_count = 0;
        for (uint32_t i = 0; i < face_count; ++i) {
            V3 vert = polytope[faces[i].a].w;
            if (dot(faces[i].normal, probe - vert) > 1e-6f) {
                visible[visible_count] = i;
                visible_count += 1;
            }
        }
        uint32_t new_count = 0;
        for (uint32_t i = 0; i < visible_count; ++i) {
            EpaFace face = faces[visible[i]];
            uint32_t edges[3][2] = {{face.a, face.b}, {face.b, face.c}, {face.c, face.a}};
            for (uint32_t e = 0; e < 3; ++e) {
                uint32_t start = edges[e][0];
                uint32_t end = edges[e][1];
                bool is_shared = false;
                for (uint32_t j = 0; j < visible_count; ++j) {
                    if (j == i) continue;
                    EpaFace other = faces[visible[j]];
                    if ((other.a == end && other.b == start) || (other.b == end && other.c == start)
                        || (other.c == end && other.a == start)) {
                        is_shared = true;
                    }
                }
                if (!is_shared && new_count < 64u) {
                    uint32_t apex = vertex_count - 1u;
                    V3 normal = cross(polytope[end].w - polytope[apex].w, polytope[start].w - polytope[apex].w);
                    float length_n = length(normal);
                    if (length_n > 1e-10f) {
                        V3 unit = normal / length_n;
                        V3 centroid = (polytope[apex].w + polytope[start].w + polytope[end].w) * (1.0f / 3.0f);
                        new_faces[new_count] = EpaFace{apex, start, end, dot(unit, centroid) > 0.0f ? -unit : unit};
                        new_count += 1;
                    }
                }
            }
        }
        uint32_t write = 0;
        uint32_t seen = 0;
        for (uint32_t i = 0; i < face_count; ++i) {
            if (seen < visible_count && visible[seen] == i) {
                seen += 1;
                continue;
            }
            faces[write] = faces[i];
            write += 1;
        }
        face_count = write;
        if (face_count + new_count > 128u) break;
        for (uint32_t i = 0; i < new_count; ++i) {
            faces[face_count] = new_faces[i];
            face_count += 1;
        }
    }
    best_dist = 3.402823466e38f;
    for (uint32_t i = 0; i < face_count; ++i) {
        float dist = dot(faces[i].normal, polytope[faces[i].a].w);
        if (dist < best_dist && length(faces[i].normal) > 0.5f) {
            best_dist = dist;
            best_face = i;
        }
    }
    EpaResult r;
    r.valid = best_dist < 3.402823466e38f;
    r.normal = faces[best_face].normal;
    r.depth = best_dist;
    r.point = polytope[faces[best_face].a].a;
    return r;
}

inline float shape_scale(const WorldShape& w) {
    float scale = w.radius + w.half_height;
    scale = fmaxw(scale, fmaxw(fmaxw(w.half_extents.x, w.half_extents.y), w.half_extents.z));
    return fmaxw(scale, 1e-4f) * fmaxw(fmaxw(w.scale.x, w.scale.y), w.scale.z);
}
inline V3 simplex_expand_dir(const SimplexPoint* s, uint32_t count) {
    if (count == 1u) return V3{1.0f, 0.0f, 0.0f};
    if (count == 2u) {
        V3 edge = s[1].w - s[0].w;
        V3 d = cross(edge, V3{1.0f, 0.0f, 0.0f});
        if (length(d) < 1e-6f) d = cross(edge, V3{0.0f, 1.0f, 0.0f});
        return normalize(d);
    }
    V3 normal = cross(s[1].w - s[0].w, s[2].w - s[0].w);
    if (length(normal) > 1e-8f) return normalize(normal);
    return V3{0.0f, 1.0f, 0.0f};
}

struct ConvexClosest {
    float distance;
    V3 point_a, point_b, normal;
    bool penetrating;
};

// convex.wgsl:464-521
inline ConvexClosest convex_closest(const Shapes& sh, const WorldShape& first, const WorldShape& second,
                                    SimplexPoint* out_simplex, uint32_t* out_count) {
    SimplexPoint simplex[4];
    uint32_t count = 0;
    ConvexClosest result;
    result.distance = 0.0f;
    result.point_a = first.center;
    result.point_b = second.center;
    result.normal = sign_normalize(second.center - first.center);
    result.penetrating = false;
    V3 dir = second.center - first.center;
    if (length(dir) < 1e-8f) dir = V3{1.0f, 0.0f, 0.0f};
    simplex[0] = support_pair(sh, first, second, dir);
    count = 1;
    SimplexResult closest = simplex_closest(simplex, count);
    float tiny = 1e-4f * fminw(shape_scale(first), shape_scale(second));
    for (uint32_t iter = 0; iter < 24u; ++iter) {
        if (closest.penetrating || length(closest.v) < tiny) {
            while (count < 4u) {
                V3 d = simplex_expand_dir(simplex, count);
                simplex[count] = support_pair(sh, first, second, d);
                count += 1;
            }
            result.penetrating = true;
            result.distance = 0.0f;
            result.point_a = closest.point_a;
            result.point_b = closest.point_b;
            break;
        }
        SimplexPoint sp = support_pair(sh, first, second, -closest.v);
        if (dot(sp.w, -closest.v) <= dot(closest.v, -closest.v) + 1e-4f * fmaxw(1.0f, dot(closest.v, closest.v))) {
            result.distance = length(closest.v);
            result.point_a = closest.point_a;
            result.point_b = closest.point_b;
            if (result.distance > 1e-6f) result.normal = sign_normalize(closest.point_b - closest.point_a);
            break;
        }
        count = simplex_reduce(simplex, closest.lambdas);
        if (simplex_holds(simplex, count, sp.w, shape_scale(second))) {
            result.distance = length(closest.v);
            result.point_a = closest.point_a;
            result.point_b = closest.point_b;
            if (result.distance > 1e-6f) result.normal = sign_normalize(closest.point_b - closest.point_a);
            break;
        }
        simplex[count] = sp;
        count += 1;
        closest = simplex_closest(simplex, count);
    }
    for (uint32_t i = 0; i < 4; ++i) out_simplex[i] = simplex[i];
    *out_count = count;
    return result;
}

struct ShapeHit {
    float distance;
    V3 point, normal;
    uint32_t triangle;
};
constexpr float kNoHit = 3.402823466e38f;

inline float support_projection_depth(const Shapes& sh, const WorldShape& f, const WorldShape& s, V3 direction) {
    V3 n = normalize(direction);
    return dot(support(sh, f, n) - support(sh, s, -n), n);
}

// convex.wgsl:532-582
inline EpaResult convex_penetration_probe(const Shapes& sh, const WorldShape& first, const WorldShape& second,
                                          const SimplexPoint* simplex, uint32_t count) {
    EpaResult best;
    best.valid = false;
    best.normal = V3{0.0f, 1.0f, 0.0f};
    best.depth = 3.402823466e38f;
    best.point = (first.center + second.center) * 0.5f;
    V3 probed[16];
    uint32_t probe_count = 0;
    for (uint32_t i = 0; i < count; ++i) {
        for (uint32_t j = i + 1; j < count; ++j) {
            for (uint32_t k = j + 1; k < count; ++k) {
                V3 normal = cross(simplex[j].w - simplex[i].w, simplex[k].w - simplex[i].w);
                if (length(normal) > 1e-8f && probe_count < 16u) {
                    probed[probe_count] = normal;
                    probe_count += 1;
                }
            }
        }
    }
    V3 center_dir = second.center - first.center;
    if (length(center_dir) > 1e-8f && probe_count < 16u) {
        probed[probe_count] = center_dir;
        probe_count += 1;
    }
    static const V3 kAxes[6] = {{1.0f, 0.0f, 0.0f}, {-1.0f, 0.0f, 0.0f}, {0.0f, 1.0f, 0.0f},
                                {0.0f, -1.0f, 0.0f}, {0.0f, 0.0f, 1.0f}, {0.0f, 0.0f, -1.0f}};
    for (uint32_t i = 0; i < 6; ++i) {
        if (probe_count < 16u) {
            probed[probe_count] = kAxes[i];
            probe_count += 1;
        }
    }
    for (uint32_t i = 0; i < probe_count; ++i) {
        float depth = support_projection_depth(sh, first, second, probed[i]);
        if (depth < best.depth) {
            best.depth = depth;
            best.normal = normalize(probed[i]);
        }
    }
    best.valid = best.depth < 3.402823466e38f;
    V3 pa = support(sh, first, best.normal);
    V3 pb = support(sh, second, -best.normal);
    best.point = (pa + pb) * 0.5f;
    return best;
}

// convex.wgsl:584-618
inline ShapeHit convex_hit(const Shapes& sh, const WorldShape& first, const WorldShape& second) {
    SimplexPoint simplex[4];
    uint32_t count = 0;
    ConvexClosest closest = convex_closest(sh, first, second, simplex, &count);
    if (!closest.penetrating) {
        EpaResult probe = convex_penetration_probe(sh, first, second, simplex, count);
        if (probe.depth > 0.0f) {
            V3 normal = probe.normal;
            if (dot(normal, second.center - first.center) < 0.0f) normal = -normal;
            return ShapeHit{-probe.depth, (closest.point_a + closest.point_b) * 0.5f, normal, DYN_NO_TRIANGLE};
        }
        if (closest.distance > 0.0f) {
            return ShapeHit{closest.distance, (closest.point_a + closest.point_b) * 0.5f, closest.normal,
                            DYN_NO_TRIANGLE};
        }
        return ShapeHit{kNoHit, splat3(0.0f), splat3(0.0f), DYN_NO_TRIANGLE};
    }
    EpaResult epa = epa_tetrahedron(sh, first, second, simplex, count);
    ShapeHit result;
    if (epa.valid && epa.depth > 0.0f && epa.depth < 3.402823466e38f && length(epa.normal) > 0.5f
        && epa.depth < support_projection_depth(sh, first, second, epa.normal)
                + 0.1f * fminw(shape_scale(first), shape_scale(second))) {
        V3 pa = support(sh, first, epa.normal);
        V3 pb = support(sh, second, -epa.normal);
        result = ShapeHit{-epa.depth, (pa + pb) * 0.5f, epa.normal, DYN_NO_TRIANGLE};
    } else {
        EpaResult probe = convex_penetration_probe(sh, first, second, simplex, count);
        V3 pa = support(sh, first, probe.normal);
        V3 pb = support(sh, second, -probe.normal);
        result = ShapeHit{-probe.depth, (pa + pb) * 0.5f, probe.normal, DYN_NO_TRIANGLE};
    }
    if (dot(result.normal, second.center - first.center) < 0.0f) result.normal = -result.normal;
    return result;
}

// ---- features: convex.wgsl:633-900 ----

constexpr uint32_t kEmptyRingFace = DYN_FEATURE_INDEX_LIMIT;
constexpr float kCapAlignment = 0.93f;
constexpr uint32_t kCylinderCapPoints = 8;
constexpr uint32_t kCylinderSidePoints = 16;
constexpr uint32_t kCylinderSideFace = 2;

inline void world_rotated_axes(const WorldShape& w, V3 axes[3]) {
    axes[0] = quat_rotate(w.rotation, V3{1.0f, 0.0f, 0.0f});
    axes[1] = quat_rotate(w.rotation, V3{0.0f, 1.0f, 0.0f});
    axes[2] = quat_rotate(w.rotation, V3{0.0f, 0.0f, 1.0f});
}
inline uint32_t box_feature_ring(const WorldShape& w, V3 direction, V3* out, uint32_t* out_ids, uint32_t* out_face) {
    V3 axes[3];
    world_rotated_axes(w, axes);
    uint32_t best_axis = 0;
    for (uint32_t i = 1; i < 3; ++i) {
        if (std::fabs(dot(axes[i], direction)) > std::fabs(dot(axes[best_axis], direction))) best_axis = i;
    }
    float sign = dot(axes[best_axis], direction) < 0.0f ? -1.0f : 1.0f;
    V3 face = axes[best_axis] * sign;
    V3 center = w.center + face * comp(w.half_extents, best_axis);
    V3 u1 = axes[(best_axis + 1u) % 3u];
    V3 u2 = axes[(best_axis + 2u) % 3u];
    float e1 = comp(w.half_extents, (best_axis + 1u) % 3u);
    float e2 = comp(w.half_extents, (best_axis + 2u) % 3u);
    out[0] = center + u1 * e1 + u2 * e2;
    out_ids[0] = box_corner_id(best_axis, sign, 1.0f, 1.0f);
    out[1] = center - u1 * e1 + u2 * e2;
    out_ids[1] = box_corner_id(best_axis, sign, -1.0f, 1.0f);
    out[2] = center - u1 * e1 - u2 * e2;
    out_ids[2] = box_corner_id(best_axis, sign, -1.0f, -1.0f);
    out[3] = center + u1 * e1 - u2 * e2;
    out_ids[3] = box_corner_id(best_axis, sign, 1.0f, -1.0f);
    *out_face = feature_field_face(best_axis * 2u + (sign > 0.0f ? 1u : 0u));
    return 4;
}
// convex.wgsl:672-721
inline uint32_t ring_of(const Shapes& sh, const WorldShape& w, V3 direction, V3* points, uint32_t* ids,
                        uint32_t count, V3* out, uint32_t* out_ids) {
    if (count <= 1u) {
        out[0] = support(sh, w, direction);
        out_ids[0] = ids[0];
        return 1;
    }
    V3 n = sign_normalize(direction);
    V3 center = splat3(0.0f);
    for (uint32_t i = 0; i < count; ++i) center = center + points[i];
    center = center / (float)count;
    V3 u;
    if (std::fabs(n.x) > 0.9f) {
        u = normalize(cross(n, V3{0.0f, 1.0f, 0.0f}));
    } else {
        u = normalize(cross(n, V3{1.0f, 0.0f, 0.0f}));
    }
    V3 v = cross(n, u);
    for (uint32_t i = 0; i < count; ++i) {
        for (uint32_t j = i + 1; j < count; ++j) {
            V3 pa = points[i] - center;
            V3 pb = points[j] - center;
            float angle_a = oatan2(dot(pa, v), dot(pa, u));
            float angle_b = oatan2(dot(pb, v), dot(pb, u));
            if (angle_b < angle_a) {
                std::swap(points[i], points[j]);
                std::swap(ids[i], ids[j]);
            }
        }
    }
    uint32_t keep = count < kFeatureMax ? count : kFeatureMax;
    for (uint32_t i = 0; i < keep; ++i) {
        out[i] = points[i];
        out_ids[i] = ids[i];
    }
    return keep;
}
// convex.wgsl:723-751 (linear path; hulls of at most 4,096 vertices)
inline uint32_t hull_feature_ring(const Shapes& sh, const WorldShape& w, V3 direction, V3* out,
                                  uint32_t* out_ids, uint32_t* out_face) {
    const dyn_shape_source_record& src = sh.sources[w.source];
    V3 d = quat_rotate(quat_conjugate(w.rotation), direction) * w.scale;
    float best_dot = dot(support_local(sh, w, d), d);
    V3 extent = rd3(src.local_max) - rd3(src.local_min);
    float eps = 1e-3f * fmaxw(fmaxw(extent.x, extent.y), extent.z) * fmaxw(fmaxw(w.scale.x, w.scale.y), w.scale.z);
    V3 points[16];
    uint32_t ids[16];
    uint32_t count = 0;
    uint32_t first_id = kEmptyRingFace;
    for (uint32_t i = 0; i < src.vertex_count && count < 16u; ++i) {
        V3 v = xyz(sh.vertices[src.vertex_offset + i]);
        if (dot(v, d) >= best_dot - eps) {
            points[count] = w.center + quat_rotate(w.rotation, v * w.scale);
            ids[count] = i;
            first_id = first_id < i ? first_id : i;
            count += 1;
        }
    }
    *out_face = feature_field_face(first_id);
    return ring_of(sh, w, direction, points, ids, count, out, out_ids);
}
// convex.wgsl:795-819
inline uint32_t capsule_feature(const WorldShape& w, V3 direction, V3* out, uint32_t* out_ids, uint32_t* out_face) {
    V3 local_direction = quat_rotate(quat_conjugate(w.rotation), direction) * w.scale;
    float cap = local_direction.y > 0.0f ? 1.0f : -1.0f;
    V3 radial = sign_normalize(local_direction) * w.radius;
    *out_face = feature_field_face(0);
    if (std::fabs(local_direction.y) > kCapAlignment * length(local_direction)) {
        V3 local = V3{0.0f, cap * w.half_height, 0.0f} + radial;
        out[0] = w.center + quat_rotate(w.rotation, local * w.scale);
        out_ids[0] = cap > 0.0f ? 1u : 0u;
        return 1;
    }
    V3 upper = V3{0.0f, w.half_height, 0.0f} + radial;
    V3 lower = V3{0.0f, -w.half_height, 0.0f} + radial;
    out[0] = w.center + quat_rotate(w.rotation, upper * w.scale);
    out[1] = w.center + quat_rotate(w.rotation, lower * w.scale);
    out_ids[0] = 0;
    out_ids[1] = 1;
    return 2;
}
// convex.wgsl:821-854
inline uint32_t cylinder_feature(const WorldShape& w, V3 direction, V3* out, uint32_t* out_ids, uint32_t* out_face) {
    V3 axis = shape_axis(w);
    float alignment = dot(axis, normalize(direction));
    if (std::fabs(alignment) > kCapAlignment) {
        float sign = alignment < 0.0f ? -1.0f : 1.0f;
        uint32_t cap = sign > 0.0f ? 1u : 0u;
        V3 cap_center = w.center + axis * w.half_height * sign;
        V3 u = normalize(cross(axis, V3{1.0f, 0.0f, 0.0f}));
        if (length(cross(axis, V3{1.0f, 0.0f, 0.0f})) < 1e-6f) u = normalize(cross(axis, V3{0.0f, 0.0f, 1.0f}));
        V3 v = cross(axis, u);
        for (uint32_t i = 0; i < kCylinderCapPoints; ++i) {
            float angle = (float)i * 0.78539816f;
            out[i] = cap_center + (u * ocos(angle) + v * osin(angle)) * w.radius;
            out_ids[i] = cap * kCylinderCapPoints + i;
        }
        *out_face = feature_field_face(cap);
        return kCylinderCapPoints;
    }
    V3 side = sign_normalize(direction - axis * dot(direction, axis));
    out[0] = w.center + axis * w.half_height + side * w.radius;
    out_ids[0] = kCylinderSidePoints;
    out[1] = w.center - axis * w.half_height + side * w.radius;
    out_ids[1] = kCylinderSidePoints + 1u;
    *out_face = feature_field_face(kCylinderSideFace);
    return 2;
}
// convex.wgsl:856-887
inline uint32_t shape_feature(const Shapes& sh, const WorldShape& w, V3 direction, V3* out, uint32_t* out_ids,
                              uint32_t* out_face, bool* ring) {
    if (w.kind == DYN_SHAPE_CUBOID) {
        *ring = true;
        return box_feature_ring(w, direction, out, out_ids, out_face);
    }
    if (w.kind == DYN_SHAPE_HULL) {
        uint32_t count = hull_feature_ring(sh, w, direction, out, out_ids, out_face);
        *ring = count > 2u;
        return count;
    }
    if (w.kind == DYN_SHAPE_CAPSULE) {
        *ring = false;
        return capsule_feature(w, direction, out, out_ids, out_face);
    }
    if (w.kind == DYN_SHAPE_CYLINDER) {
        uint32_t count = cylinder_feature(w, direction, out, out_ids, out_face);
        *ring = count > 2u;
        return count;
    }
    *ring = false;
    out[0] = support(sh, w, direction);
    out_ids[0] = 0;
    *out_face = feature_field_face(0);
    return 1;
}
inline float feature_radius(const V3* points, uint32_t count) {
    V3 center = splat3(0.0f);
    for (uint32_t i = 0; i < count; ++i) center = center + points[i];
    center = center / (float)count;
    float radius = 0.0f;
    for (uint32_t i = 0; i < count; ++i) radius = fmaxw(radius, length(points[i] - center));
    return radius;
}

constexpr uint32_t kClipPoints = kManifoldCandidates;

// convex.wgsl:910-982
inline uint32_t clip_feature_to_ring(const V3* points, const uint32_t* ids, uint32_t count, const V3* ring,
                                     uint32_t ring_count, V3 ref_dir, V3* out_points, uint32_t* out_ids) {
    V3 held_points[kClipPoints];
    uint32_t held_ids[kClipPoints];
    for (uint32_t i = 0; i < count; ++i) {
        held_points[i] = points[i];
        held_ids[i] = ids[i];
    }
    uint32_t live = count;
    for (uint32_t side = 0; side < ring_count; ++side) {
        V3 current = ring[side];
        V3 next = ring[(side + 1u) % ring_count];
        V3 plane_normal = normalize(cross(next - current, ref_dir));
        V3 kept_points[kClipPoints];
        uint32_t kept_ids[kClipPoints];
        uint32_t written = 0;
        if (live == 2u) {
            V3 fp = held_points[0];
            V3 sp = held_points[1];
            float first_side = dot(fp - current, plane_normal) - kClipMargin;
            float second_side = dot(sp - current, plane_normal) - kClipMargin;
            if (first_side <= 0.0f) {
                kept_points[written] = fp;
                kept_ids[written] = held_ids[0];
                written += 1;
            }
            if (first_side * second_side < 0.0f && written < kClipPoints) {
                kept_points[written] = fp + (sp - fp) * (first_side / (first_side - second_side));
                kept_ids[written] = feature_field_clip(side * kClipPoints);
                written += 1;
            }
            if (second_side <= 0.0f && written < kClipPoints) {
                kept_points[written] = sp;
                kept_ids[written] = held_ids[1];
                written += 1;
            }
        } else {
            for (uint32_t i = 0; i < live; ++i) {
                V3 cp = held_points[i];
                V3 np = held_points[(i + 1u) % live];
                float cs = dot(cp - current, plane_normal) - kClipMargin;
                float ns = dot(np - current, plane_normal) - kClipMargin;
                if (cs <= 0.0f && written < kClipPoints) {
                    kept_points[written] = cp;
                    kept_ids[written] = held_ids[i];
                    written += 1;
                }
                if (cs * ns < 0.0f && written < kClipPoints) {
                    kept_points[written] = cp + (np - cp) * (cs / (cs - ns));
                    kept_ids[written] = feature_field_clip(side * kClipPoints + i);
                    written += 1;
                }
            }
        }
        live = written;
        for (uint32_t i = 0; i < written; ++i) {
            held_points[i] = kept_points[i];
            held_ids[i] = kept_ids[i];
        }
        if (live == 0u) break;
    }
    for (uint32_t i = 0; i < live; ++i) {
        out_points[i] = held_points[i];
        out_ids[i] = held_ids[i];
    }
    return live;
}

// convex.wgsl:984-1071
inline bool convex_pair_manifold(const Shapes& sh, const WorldShape& first, const WorldShape& second, V3 direction,
                                 Manifold* m) {
    V3 first_points[kFeatureMax], second_points[kFeatureMax];
    uint32_t first_ids[kFeatureMax], second_ids[kFeatureMax];
    uint32_t first_face = 0, second_face = 0;
    bool first_ring = false, second_ring = false;
    uint32_t first_count = shape_feature(sh, first, direction, first_points, first_ids, &first_face, &first_ring);
    uint32_t second_count = shape_feature(sh, second, -direction, second_points, second_ids, &second_face, &second_ring);
    if (!first_ring && !second_ring) return false;
    bool first_reference = first_ring;
    if (first_ring && second_ring) {
        first_reference = feature_radius(first_points, first_count) >= feature_radius(second_points, second_count);
    }
    const V3* reference;
    uint32_t reference_count;
    uint32_t reference_face = second_face;
    const V3* incident;
    const uint32_t* incident_ids;
    uint32_t incident_count;
    V3 ref_dir;
    if (first_reference) {
        reference = first_points;
        reference_count = first_count;
        reference_face = first_face;
        incident = second_points;
        incident_ids = second_ids;
        incident_count = second_count;
        ref_dir = direction;
    } else {
        reference = second_points;
        reference_count = second_count;
        incident = first_points;
        incident_ids = first_ids;
        incident_count = first_count;
        ref_dir = -direction;
    }
    V3 center = splat3(0.0f);
    for (uint32_t i = 0; i < reference_count; ++i) center = center + reference[i];
    center = center / (float)reference_count;
    V3 deepest = splat3(0.0f);
    float deepest_depth = -1e30f;
    for (uint32_t i = 0; i < incident_count; ++i) {
        float depth = dot(center - incident[i], ref_dir);
        if (depth > deepest_depth) {
            deepest_depth = depth;
            deepest = incident[i];
        }
    }
    V3 clipped_points[kClipPoints];
    uint32_t clipped_ids[kClipPoints];
    uint32_t clipped = clip_feature_to_ring(incident, incident_ids, incident_count, reference, reference_count,
                                            ref_dir, clipped_points, clipped_ids);
    Candidate candidates[kManifoldCandidates];
    uint32_t candidate_count = 0;
    for (uint32_t i = 0; i < clipped && candidate_count < kManifoldCandidates; ++i) {
        float depth = dot(center - clipped_points[i], ref_dir);
        if (depth > 0.0f) {
            candidates[candidate_count] = Candidate{
                clipped_points[i] - ref_dir * (depth * 0.5f), depth,
                first_reference ? feature_vertex(reference_face, clipped_ids[i])
                                : feature_vertex(clipped_ids[i], reference_face)};
            candidate_count += 1;
        }
    }
    if (candidate_count == 0u) {
        if (deepest_depth <= 0.0f) return false;
        manifold_push(m, deepest - ref_dir * (deepest_depth * 0.5f), deepest_depth, DYN_FEATURE_POINT);
        return true;
    }
    manifold_keep(m, candidates, candidate_count);
    return true;
}

// narrowphase.wgsl:485-512
inline Manifold plane_convex(const Shapes& sh, const WorldShape& plane, const WorldShape& convex, float margin) {
    Manifold m;
    V3 n = quat_rotate(plane.rotation, V3{0.0f, 1.0f, 0.0f});
    float center_side = dot(convex.center - plane.center, n);
    V3 facing = center_side < 0.0f ? -n : n;
    manifold_emit(&m, facing);
    V3 points[kFeatureMax];
    uint32_t ids[kFeatureMax];
    uint32_t feature = 0;
    bool ring = false;
    uint32_t count = shape_feature(sh, convex, -facing, points, ids, &feature, &ring);
    Candidate candidates[kManifoldCandidates];
    uint32_t candidate_count = 0;
    for (uint32_t i = 0; i < count; ++i) {
        float depth = dot(plane.center - points[i], facing);
        if (depth <= -margin) continue;
        candidates[candidate_count] = Candidate{points[i] + facing * (depth * 0.5f), depth,
                                                feature_vertex(feature_field_face(0), ids[i])};
        candidate_count += 1;
    }
    manifold_keep(&m, candidates, candidate_count);
    return m;
}

inline void manifold_from_hit(Manifold* m, const ShapeHit& hit, float margin) {
    if (hit.distance <= margin) manifold_push(m, hit.point, -hit.distance, DYN_FEATURE_POINT);
}
inline bool scaled_shape(const dyn_collider_record& c) {
    return c.scale[0] != 1.0f || c.scale[1] != 1.0f || c.scale[2] != 1.0f;
}

// core.wgsl:302-313
inline float material_combine(float first, float second, uint32_t mode) {
    if (mode == 1u) return fminw(first, second);
    if (mode == 2u) return fmaxw(first, second);
    if (mode == 3u) return (first + second) * 0.5f;
    return std::sqrt(first * second);
}

}  // namespace orc
