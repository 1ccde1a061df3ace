// narrow.cuh - contact manifold generation on sm_100a (one thread per candidate pair).
//
// Restates crates/dynamis-rigid/shaders/narrowphase.wgsl (pair kernels), and the shape, GJK,
// EPA, probe and feature-clipping functions of crates/dynamis-shader/shaders/convex.wgsl and
// core.wgsl, over the device's structure-of-arrays collider tables and 128-byte body rows.
// Operand order follows the WGSL so results are reproducible bit for bit (see dmath.cuh).
// World geometry other than planes and hulls above 4,096 vertices are outside this path.
#pragma once

#include "dmath.cuh"
#include "layout.cuh"

namespace dyn {

struct DBody {
    f3 position;
    float4 orientation;
    f3 velocity;
    f3 angular_velocity;
    float inverse_mass;
    uint32_t flags;
    uint32_t sleeping;
    f3 com;
    float4 ii0;
    float2 ii1;
};

__device__ __forceinline__ DBody load_dbody(const BodyHot* hot, uint32_t row) {
    const BodyHot& h = hot[row];
    float4 p = h.pos, q = h.rot, v = h.vel, w = h.ang, c = h.com, i0 = h.ii0, i1 = h.ii1;
    uint4 aux = h.aux;
    DBody b;
    b.position = xyz(p);
    b.inverse_mass = p.w;
    b.orientation = q;
    b.velocity = xyz(v);
    b.angular_velocity = xyz(w);
    b.com = xyz(c);
    b.ii0 = i0;
    b.ii1 = make_float2(i1.x, i1.y);
    b.sleeping = aux.x;
    b.flags = aux.y;
    return b;
}

DYN_HD bool kinematic_flag(uint32_t flags) { return (flags & 1u) != 0u; }
DYN_HD bool simulates(float im, uint32_t flags) { return !kinematic_flag(flags) && im > 0.0f; }
DYN_HD bool moves(float im, uint32_t flags) { return kinematic_flag(flags) || im > 0.0f; }
__device__ __forceinline__ bool dbody_inert(const DBody& b) { return !simulates(b.inverse_mass, b.flags) || b.sleeping != 0u; }
__device__ __forceinline__ DBody dbody_frozen(DBody b) {
    b.inverse_mass = 0.0f;
    b.ii0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    b.ii1 = make_float2(0.0f, 0.0f);
    return b;
}
__device__ __forceinline__ f3 dbody_com(const DBody& b) { return b.position + quat_rotate(b.orientation, b.com); }
__device__ __forceinline__ f3 inv_inertia_world(float4 i0, float2 i1, float4 q, f3 v) {
    f3 local = quat_rotate(quat_conj(q), v);
    return quat_rotate(q, sym_apply(i0, i1, local));
}
__device__ __forceinline__ f3 dbody_iinv(const DBody& b, f3 v) { return inv_inertia_world(b.ii0, b.ii1, b.orientation, v); }
__device__ __forceinline__ f3 point_velocity(const DBody& b, f3 p) {
    return b.velocity + cross(b.angular_velocity, p - dbody_com(b));
}
__device__ __forceinline__ f3 relative_velocity(const DBody& a, const DBody& b, f3 pa, f3 pb) {
    return point_velocity(b, pb) - point_velocity(a, pa);
}

// A collider placed in the world (core.wgsl:34-43, 473-484).
struct WShape {
    uint32_t kind;
    uint32_t source;
    float radius;
    float half_height;
    f3 center;
    f3 half_extents;
    float4 rotation;
    f3 scale;
};

struct DColl {
    uint32_t kind, flags, source;
    f3 offset;
    float radius;
    float4 lrot;
    f3 half_extents;
    float half_height;
    f3 scale;
};

__device__ __forceinline__ DColl load_dcoll(const DeviceWorld& w, uint32_t slot) {
    DColl c;
    uint4 k = w.c_kind[slot];
    float4 o = w.c_offset[slot], h = w.c_half[slot], s = w.c_scale[slot];
    c.kind = k.x;
    c.flags = k.y;
    c.source = k.z;
    c.offset = xyz(o);
    c.radius = o.w;
    c.lrot = w.c_lrot[slot];
    c.half_extents = xyz(h);
    c.half_height = h.w;
    c.scale = xyz(s);
    return c;
}
__device__ __forceinline__ WShape world_shape(f3 position, float4 orientation, const DColl& c) {
    WShape s;
    s.kind = c.kind;
    s.radius = c.radius;
    s.half_height = c.half_height;
    s.center = position + quat_rotate(orientation, c.offset);
    s.half_extents = c.half_extents;
    s.rotation = quat_mul(orientation, c.lrot);
    s.source = c.source;
    s.scale = c.scale;
    return s;
}

DYN_HD bool shape_world_geometry(uint32_t k) { return k == 6u || k == 7u || k == 9u; }
DYN_HD bool shape_analytic(uint32_t k) { return k == 1u || k == 2u || k == 3u; }
DYN_HD bool shape_has_source(uint32_t k) { return k == 5u || k == 6u || k == 7u || k == 8u; }

struct DAabb {
    f3 min, max;
};

// core.wgsl:490-536
__device__ __forceinline__ DAabb world_aabb(const DeviceWorld& w, const WShape& s) {
    if (s.kind == 9u) {
        return DAabb{s.center - s3(1e6f), s.center + s3(1e6f)};
    }
    if (shape_has_source(s.kind)) {
        const dyn_shape_source_record& src = w.sources[s.source];
        f3 smin = mk3(src.local_min[0], src.local_min[1], src.local_min[2]) * s.scale;
        f3 smax = mk3(src.local_max[0], src.local_max[1], src.local_max[2]) * s.scale;
        f3 center = s.center + quat_rotate(s.rotation, (smin + smax) * 0.5f);
        f3 half = (smax - smin) * 0.5f;
        f3 extent = vabs(quat_rotate(s.rotation, mk3(half.x, 0.0f, 0.0f)))
            + vabs(quat_rotate(s.rotation, mk3(0.0f, half.y, 0.0f)))
            + vabs(quat_rotate(s.rotation, mk3(0.0f, 0.0f, half.z)));
        return DAabb{center - extent, center + extent};
    }
    f3 extent = s3(0.0f);
    if (s.kind == 1u) {
        extent = s3(s.radius);
    } else if (s.kind == 2u) {
        f3 e = s.half_extents;
        extent = vabs(quat_rotate(s.rotation, mk3(e.x, 0.0f, 0.0f))) + vabs(quat_rotate(s.rotation, mk3(0.0f, e.y, 0.0f)))
            + vabs(quat_rotate(s.rotation, mk3(0.0f, 0.0f, e.z)));
    } else if (s.kind == 3u || s.kind == 4u) {
        f3 axis = quat_rotate(s.rotation, mk3(0.0f, 1.0f, 0.0f));
        extent = vabs(axis * s.half_height) + s3(s.radius);
    }
    float m = wmax(wmax(s.scale.x, s.scale.y), s.scale.z);
    extent = extent * m;
    return DAabb{s.center - extent, s.center + extent};
}

// ---- manifold candidates (core.wgsl:614-760) ----
constexpr uint32_t kFeatPoint = 0u;
constexpr uint32_t kFeatVertex = 1u << 28;
constexpr uint32_t kFeatEdge = 2u << 28;
constexpr uint32_t kFeatFace = 3u << 28;
constexpr uint32_t kFeatClip = 1u << 12;
constexpr uint32_t kFeatFaceBit = 1u << 13;
constexpr float kClipMargin = 1e-4f;

DYN_HD uint32_t feature_pair(uint32_t kind, uint32_t f, uint32_t s) { return kind | (f << 14) | s; }
DYN_HD uint32_t feature_mirror(uint32_t feature) {
    uint32_t kind = feature & 0xF0000000u;
    if (kind == kFeatPoint) return feature;
    uint32_t first = (feature >> 14) & 0x3FFFu;
    uint32_t second = feature & 0x3FFFu;
    return kind | (second << 14) | first;
}

struct Cand {
    f3 position;
    float depth;
    uint32_t feature;
};
struct Mani {
    uint32_t count;
    f3 normal;
    Cand p[4];
};
__device__ __forceinline__ void mani_emit(Mani* m, f3 normal) {
    m->count = 0;
    m->normal = normal;
}
__device__ __forceinline__ void mani_push(Mani* m, f3 point, float depth, uint32_t feature) {
    if (m->count >= 4u) return;
    m->p[m->count] = Cand{point, depth, feature};
    m->count += 1;
}
__device__ __forceinline__ void cand_swap(Cand* c, uint32_t a, uint32_t b) {
    Cand t = c[a];
    c[a] = c[b];
    c[b] = t;
}
__device__ __forceinline__ float mani_gap(const Cand* c, uint32_t kept, uint32_t index) {
    float gap = 3.402823466e38f;
    for (uint32_t held = 0; held < kept; ++held) gap = wmin(gap, length(c[index].position - c[held].position));
    return gap;
}
__device__ void mani_keep(Mani* m, Cand* c, uint32_t count) {
    uint32_t lead = 0;
    for (uint32_t i = 1; i < count; ++i) {
        float depth = c[i].depth, held = c[lead].depth;
        if (depth > held || (depth == held && c[i].feature < c[lead].feature)) lead = i;
    }
    cand_swap(c, 0, lead);
    for (uint32_t kept = 1; kept < count; ++kept) {
        uint32_t best = kept;
        float best_gap = mani_gap(c, kept, kept);
        for (uint32_t i = kept + 1; i < count; ++i) {
            float gap = mani_gap(c, kept, i);
            if (gap > best_gap) {
                best_gap = gap;
                best = i;
            }
        }
        if (best != kept) cand_swap(c, kept, best);
    }
    for (uint32_t i = 0; i < count && m->count < 4u; ++i) mani_push(m, c[i].position, c[i].depth, c[i].feature);
}

// ---- analytic kernels (narrowphase.wgsl:33-473) ----
__device__ __forceinline__ f3 coll_center(const DBody& b, const DColl& c) { return b.position + quat_rotate(b.orientation, c.offset); }
__device__ __forceinline__ void coll_axes(const DBody& b, const DColl& c, f3 axes[3]) {
    float4 q = quat_mul(b.orientation, c.lrot);
    axes[0] = quat_rotate(q, mk3(1.0f, 0.0f, 0.0f));
    axes[1] = quat_rotate(q, mk3(0.0f, 1.0f, 0.0f));
    axes[2] = quat_rotate(q, mk3(0.0f, 0.0f, 1.0f));
}

__device__ Mani sphere_sphere(const DBody& fb, const DColl& fc, const DBody& sb, const DColl& sc, float margin) {
    Mani m;
    f3 fcen = coll_center(fb, fc), scen = coll_center(sb, sc);
    f3 delta = scen - fcen;
    float distance = length(delta);
    f3 normal = sign_normalize(delta);
    if (distance <= 1e-6f) {
        f3 rel = relative_velocity(fb, sb, scen, fcen);
        if (length(rel) > 1e-6f) normal = -normalize(rel);
    }
    mani_emit(&m, normal);
    float rsum = fc.radius + sc.radius;
    if (distance > rsum + margin) return m;
    float depth = rsum - distance;
    mani_push(&m, fcen + normal * (fc.radius - depth * 0.5f), depth, kFeatPoint);
    return m;
}

__device__ Mani sphere_box(const DBody& sph, const DColl& scol, const DBody& box, const DColl& bcol, float margin) {
    Mani m;
    f3 center = sph.position + quat_rotate(sph.orientation, scol.offset);
    float4 q = quat_mul(box.orientation, bcol.lrot);
    f3 bcen = coll_center(box, bcol);
    f3 local = quat_rotate(quat_conj(q), center - bcen);
    f3 clamped = vclamp(local, -bcol.half_extents, bcol.half_extents);
    f3 closest = coll_center(box, bcol) + quat_rotate(q, clamped);
    f3 delta = closest - center;
    float distance = length(delta);
    f3 normal = sign_normalize(delta);
    float depth = scol.radius - distance;
    if (distance <= 1e-6f) {
        // box_nearest_face (narrowphase.wgsl:65-83)
        f3 l2 = quat_rotate(quat_conj(q), center - coll_center(box, bcol));
        f3 clearance = bcol.half_extents - vabs(l2);
        f3 ac = vabs(clearance);
        uint32_t axis = (ac.x < ac.y && ac.x < ac.z) ? 0u : (ac.y < ac.z ? 1u : 2u);
        f3 facing = s3(0.0f);
        if (axis == 0u) facing = mk3(l2.x > 0.0f ? -1.0f : 1.0f, 0.0f, 0.0f);
        else if (axis == 1u) facing = mk3(0.0f, l2.y > 0.0f ? -1.0f : 1.0f, 0.0f);
        else facing = mk3(0.0f, 0.0f, l2.z > 0.0f ? -1.0f : 1.0f);
        f3 face_normal = -quat_rotate(q, facing);
        normal = -face_normal;
        depth = scol.radius + comp(clearance, axis);
    }
    mani_emit(&m, normal);
    if (depth <= -margin) return m;
    mani_push(&m, closest - normal * (depth * 0.5f), depth, kFeatPoint);
    return m;
}

__device__ __forceinline__ void capsule_segment(const DBody& b, const DColl& c, f3* s0, f3* s1) {
    float4 q = quat_mul(b.orientation, c.lrot);
    f3 axis = quat_rotate(q, mk3(0.0f, 1.0f, 0.0f));
    f3 center = coll_center(b, c);
    *s0 = center - axis * c.half_height;
    *s1 = center + axis * c.half_height;
}
__device__ Mani sphere_capsule(const DBody& sph, const DColl& scol, const DBody& cap, const DColl& ccol, float margin) {
    Mani m;
    f3 s0, s1;
    capsule_segment(cap, ccol, &s0, &s1);
    f3 center = sph.position + quat_rotate(sph.orientation, scol.offset);
    f3 ab = s1 - s0;
    f3 closest = s0;
    float denom = dot(ab, ab);
    if (!(denom < 1e-10f)) {
        float t = wclamp(dot(center - s0, ab) / denom, 0.0f, 1.0f);
        closest = s0 + ab * t;
    }
    f3 delta = closest - center;
    float distance = length(delta);
    float rsum = scol.radius + ccol.radius;
    mani_emit(&m, sign_normalize(delta));
    if (distance > rsum + margin) return m;
    f3 normal = sign_normalize(delta);
    float depth = rsum - distance;
    mani_push(&m, closest - normal * (depth * 0.5f), depth, kFeatPoint);
    return m;
}
__device__ Mani capsule_capsule(const DBody& fb, const DColl& fc, const DBody& sb, const DColl& sc, float margin) {
    Mani m;
    f3 a0, a1, b0, b1;
    capsule_segment(fb, fc, &a0, &a1);
    capsule_segment(sb, sc, &b0, &b1);
    f3 d1 = a1 - a0, d2 = b1 - b0, r = a0 - b0;
    float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    float s = 0.0f, t = 0.0f;
    if (a <= 1e-10f && e <= 1e-10f) {
    } else if (a <= 1e-10f) {
        t = wclamp(f / e, 0.0f, 1.0f);
    } else {
        float c = dot(d1, r);
        if (e <= 1e-10f) {
            t = 0.0f;
            s = wclamp(-c / a, 0.0f, 1.0f);
        } else {
            float b = dot(d1, d2);
            float denom = a * e - b * b;
            s = denom != 0.0f ? wclamp((b * f - c * e) / denom, 0.0f, 1.0f) : 0.0f;
            t = (b * s + f) / e;
            if (t < 0.0f) {
                t = 0.0f;
                s = wclamp(-c / a, 0.0f, 1.0f);
            } else if (t > 1.0f) {
                t = 1.0f;
                s = wclamp((b - c) / a, 0.0f, 1.0f);
            }
        }
    }
    f3 cs = a0 + d1 * s, ce = b0 + d2 * t;
    f3 delta = ce - cs;
    float distance = length(delta);
    float rsum = fc.radius + sc.radius;
    mani_emit(&m, sign_normalize(delta));
    if (distance > rsum + margin) return m;
    mani_push(&m, (cs + ce) * 0.5f, rsum - distance, kFeatPoint);
    return m;
}

DYN_HD uint32_t box_corner_id(uint32_t axis, float sign, float first, float second) {
    uint32_t id = 0;
    id |= sign > 0.0f ? (1u << axis) : 0u;
    id |= first > 0.0f ? (1u << ((axis + 1u) % 3u)) : 0u;
    id |= second > 0.0f ? (1u << ((axis + 2u) % 3u)) : 0u;
    return id;
}

struct BoxGeo {
    f3 axes[3];
    f3 half;
    f3 center;
};
__device__ __forceinline__ BoxGeo box_geo(const DBody& b, const DColl& c) {
    BoxGeo g;
    coll_axes(b, c, g.axes);
    g.half = c.half_extents;
    g.center = coll_center(b, c);
    return g;
}
__device__ __forceinline__ float support_radius(const BoxGeo& g, f3 axis) {
    return fabsf(dot(g.axes[0], axis)) * g.half.x + fabsf(dot(g.axes[1], axis)) * g.half.y
        + fabsf(dot(g.axes[2], axis)) * g.half.z;
}
__device__ __forceinline__ f3 box_support_geo(const BoxGeo& g, f3 direction) {
    f3 point = g.center;
    for (uint32_t i = 0; i < 3; ++i) {
        float h = comp(g.half, i);
        point = point + g.axes[i] * (dot(g.axes[i], direction) > 0.0f ? h : -h);
    }
    return point;
}
// narrowphase.wgsl:215-252 (box_face), on a box's geometry
__device__ f3 box_face_geo(const BoxGeo& g, f3 face_normal, f3 corners[4], uint32_t ids[4], uint32_t* out_face) {
    uint32_t axis = 0;
    for (uint32_t i = 1; i < 3; ++i) {
        if (fabsf(dot(face_normal, g.axes[i])) > fabsf(dot(face_normal, g.axes[axis]))) axis = i;
    }
    float sign = dot(face_normal, g.axes[axis]) < 0.0f ? -1.0f : 1.0f;
    f3 n = g.axes[axis] * sign;
    f3 u = g.axes[(axis + 1u) % 3u];
    f3 v = g.axes[(axis + 2u) % 3u];
    float hu = comp(g.half, (axis + 1u) % 3u);
    float hv = comp(g.half, (axis + 2u) % 3u);
    f3 fc = g.center + n * comp(g.half, axis);
    corners[0] = fc + (u * hu + v * hv);
    corners[1] = fc + (-u * hu + v * hv);
    corners[2] = fc + (-u * hu - v * hv);
    corners[3] = fc + (u * hu - v * hv);
    ids[0] = box_corner_id(axis, sign, 1.0f, 1.0f);
    ids[1] = box_corner_id(axis, sign, -1.0f, 1.0f);
    ids[2] = box_corner_id(axis, sign, -1.0f, -1.0f);
    ids[3] = box_corner_id(axis, sign, 1.0f, -1.0f);
    *out_face = axis * 2u + (sign > 0.0f ? 1u : 0u);
    return fc;
}
__device__ uint32_t clip_polygon(const f3* pts, const uint32_t* ids, uint32_t count, f3 pp, f3 pn, uint32_t group,
                                 uint32_t side, f3* out_p, uint32_t* out_i) {
    uint32_t oc = 0;
    for (uint32_t i = 0; i < count; ++i) {
        f3 cur = pts[i];
        f3 nxt = pts[(i + 1u) % count];
        float cd = dot(cur - pp, pn) - kClipMargin;
        float nd = dot(nxt - pp, pn) - kClipMargin;
        if (cd <= 0.0f && oc < 8u) {
            out_p[oc] = cur;
            out_i[oc] = ids[i];
            oc += 1;
        }
        if (cd * nd < 0.0f) {
            float t = cd / (cd - nd);
            if (oc < 8u) {
                out_p[oc] = cur + (nxt - cur) * t;
                out_i[oc] = kFeatClip | (group * 32u + side * 8u + i);
                oc += 1;
            }
        }
    }
    return oc;
}

// narrowphase.wgsl:325-473
__device__ Mani box_box_sat(const DBody& fb, const DColl& fc, const DBody& sb, const DColl& sc, float margin) {
    Mani m;
    m.count = 0;
    m.normal = s3(0.0f);
    BoxGeo L = box_geo(fb, fc);
    BoxGeo R = box_geo(sb, sc);
    f3 delta = R.center - L.center;
    float face_depth = 1e30f;
    f3 face_axis = L.axes[0];
    bool face_on_right = false;
    for (uint32_t i = 0; i < 3; ++i) {
        f3 ax = L.axes[i];
        float overlap = comp(L.half, i) + support_radius(R, ax) - fabsf(dot(delta, ax));
        if (overlap < face_depth) {
            face_depth = overlap;
            face_axis = ax;
            face_on_right = false;
        }
        f3 bx = R.axes[i];
        float other = comp(R.half, i) + support_radius(L, bx) - fabsf(dot(delta, bx));
        if (other < face_depth) {
            face_depth = other;
            face_axis = bx;
            face_on_right = true;
        }
    }
    // No contact whatever the edge axes give: an edge axis wins only when its depth is below the face
    // depth (edge_depth <= edge_depth + 1e-3 * extent < face_depth, rounding being monotone), and
    // either depth at or below -margin answers no contact below. So the nine edge axes are skipped.
    if (face_depth <= -margin) return m;
    float edge_depth = 1e30f;
    f3 edge_axis = face_axis;
    uint32_t efa = 0, esa = 0;
    for (uint32_t i = 0; i < 3; ++i) {
        for (uint32_t j = 0; j < 3; ++j) {
            f3 crossed = cross(L.axes[i], R.axes[j]);
            float len = length(crossed);
            if (len < 1e-8f) continue;
            f3 axis = crossed / len;
            float overlap = support_radius(L, axis) + support_radius(R, axis) - fabsf(dot(delta, axis));
            if (overlap < edge_depth) {
                edge_depth = overlap;
                edge_axis = axis;
                efa = i;
                esa = j;
            }
        }
    }
    float extent = wmax(wmax(L.half.x, L.half.y), L.half.z) + wmax(wmax(R.half.x, R.half.y), R.half.z);
    bool edge_sep = edge_depth + 1e-3f * extent < face_depth;
    float depth = edge_sep ? edge_depth : face_depth;
    if (depth <= -margin) return m;
    f3 axis = edge_sep ? edge_axis : face_axis;
    f3 sgn = dot(axis, delta) < 0.0f ? -axis : axis;
    mani_emit(&m, sgn);
    if (edge_sep) {
        f3 point = (box_support_geo(L, sgn) + box_support_geo(R, -sgn)) * 0.5f;
        mani_push(&m, point, depth, feature_pair(kFeatEdge, efa, esa));
        return m;
    }
    const BoxGeo& ref = face_on_right ? R : L;
    const BoxGeo& inc = face_on_right ? L : R;
    f3 ref_normal = face_on_right ? -sgn : sgn;
    f3 ref_corners[4];
    uint32_t ref_ids[4];
    uint32_t ref_face = 0;
    f3 ref_center = box_face_geo(ref, ref_normal, ref_corners, ref_ids, &ref_face);
    uint32_t ia = 0;
    for (uint32_t i = 1; i < 3; ++i) {
        if (fabsf(dot(inc.axes[i], ref_normal)) > fabsf(dot(inc.axes[ia], ref_normal))) ia = i;
    }
    f3 inc_normal = inc.axes[ia] * (dot(inc.axes[ia], ref_normal) > 0.0f ? -1.0f : 1.0f);
    f3 inc_corners[4];
    uint32_t inc_ids[4];
    uint32_t inc_face = 0;
    box_face_geo(inc, inc_normal, inc_corners, inc_ids, &inc_face);
    uint32_t ref_field = kFeatFaceBit | ref_face;
    f3 pa[8], pb[8];
    uint32_t ida[8], idb[8];
    for (uint32_t i = 0; i < 4; ++i) {
        pa[i] = inc_corners[i];
        ida[i] = inc_ids[i];
    }
    uint32_t pc = 4;
    for (uint32_t side = 0; side < 4; ++side) {
        f3 cur = ref_corners[side];
        f3 nxt = ref_corners[(side + 1u) % 4u];
        f3 pn = normalize(cross(nxt - cur, ref_normal));
        if (side % 2u == 0u) {
            pc = clip_polygon(pa, ida, pc, cur, pn, inc_face, side, pb, idb);
        } else {
            pc = clip_polygon(pb, idb, pc, cur, pn, inc_face, side, pa, ida);
        }
        if (pc == 0u) break;
    }
    Cand cands[16];
    uint32_t cc = 0;
    for (uint32_t i = 0; i < pc && cc < 16u; ++i) {
        float pd = dot(ref_center - pa[i], ref_normal);
        if (pd >= -margin) {
            cands[cc] = Cand{pa[i] - ref_normal * (pd * 0.5f), pd,
                             face_on_right ? feature_pair(kFeatFace, ida[i], ref_field) : feature_pair(kFeatFace, ref_field, ida[i])};
            cc += 1;
        }
    }
    if (cc == 0u) {
        for (uint32_t i = 0; i < 4 && cc < 16u; ++i) {
            float pd = dot(ref_center - inc_corners[i], ref_normal);
            if (pd >= -margin) {
                cands[cc] = Cand{inc_corners[i] - ref_normal * (pd * 0.5f), pd,
                                 face_on_right ? feature_pair(kFeatFace, inc_ids[i], ref_field)
                                               : feature_pair(kFeatFace, ref_field, inc_ids[i])};
                cc += 1;
            }
        }
    }
    if (cc == 0u) {
        mani_push(&m, ref_center - ref_normal * (face_depth * 0.5f), face_depth, kFeatPoint);
        return m;
    }
    mani_keep(&m, cands, cc);
    return m;
}

// ---- convex support maps (convex.wgsl:1-91) ----
__device__ f3 support_local(const DeviceWorld& w, const WShape& s, f3 d) {
    if (s.kind == 1u) return normalize(d) * s.radius;
    if (s.kind == 2u) {
        f3 signs = mk3(d.x > 0.0f ? 1.0f : -1.0f, d.y > 0.0f ? 1.0f : -1.0f, d.z > 0.0f ? 1.0f : -1.0f);
        return signs * s.half_extents;
    }
    if (s.kind == 3u) {
        f3 tip = mk3(0.0f, 1.0f, 0.0f) * s.half_height * (d.y > 0.0f ? 1.0f : -1.0f);
        return tip + normalize(d) * s.radius;
    }
    if (s.kind == 4u) {
        f3 base = mk3(0.0f, 1.0f, 0.0f) * s.half_height * (d.y > 0.0f ? 1.0f : -1.0f);
        f3 radial = d - mk3(0.0f, d.y, 0.0f);
        if (length(radial) < 1e-6f) return base;
        return base + normalize(radial) * s.radius;
    }
    const dyn_shape_source_record& src = w.sources[s.source];
    const float4* verts = w.vertices + src.vertex_offset;
    const uint32_t count = src.vertex_count;
    float best_dot = -3.402823466e38f;
    f3 best = s3(0.0f);
    // four loads in flight, then the same comparisons in index order as the one-at-a-time scan
    uint32_t i = 0;
    for (; i + 4u <= count; i += 4u) {
        const f3 v0 = xyz(__ldg(verts + i)), v1 = xyz(__ldg(verts + i + 1u));
        const f3 v2 = xyz(__ldg(verts + i + 2u)), v3 = xyz(__ldg(verts + i + 3u));
        const float s0 = dot(v0, d), s1 = dot(v1, d), s2 = dot(v2, d), s3_ = dot(v3, d);
        if (s0 > best_dot) { best_dot = s0; best = v0; }
        if (s1 > best_dot) { best_dot = s1; best = v1; }
        if (s2 > best_dot) { best_dot = s2; best = v2; }
        if (s3_ > best_dot) { best_dot = s3_; best = v3; }
    }
    for (; i < count; ++i) {
        const f3 v = xyz(__ldg(verts + i));
        const float sd = dot(v, d);
        if (sd > best_dot) {
            best_dot = sd;
            best = v;
        }
    }
    return best;
}
__device__ __forceinline__ f3 support(const DeviceWorld& w, const WShape& s, f3 direction) {
    f3 local_d = quat_rotate(quat_conj(s.rotation), direction);
    f3 local = support_local(w, s, local_d * s.scale);
    return s.center + quat_rotate(s.rotation, local * s.scale);
}

// ---- GJK (convex.wgsl:93-278, 439-521) ----
struct SPt {
    f3 w, a, b;
};
__device__ f3 closest_on_triangle(f3 a, f3 b, f3 c, f3* wts) {
    f3 origin = s3(0.0f);
    f3 ab = b - a, ac = c - a, ap = origin - a;
    float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) {
        *wts = mk3(1.0f, 0.0f, 0.0f);
        return a;
    }
    f3 bp = origin - b;
    float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) {
        *wts = mk3(0.0f, 1.0f, 0.0f);
        return b;
    }
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float t = d1 / (d1 - d3);
        *wts = mk3(1.0f - t, t, 0.0f);
        return a + ab * t;
    }
    f3 cp = origin - c;
    float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) {
        *wts = mk3(0.0f, 0.0f, 1.0f);
        return c;
    }
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        float t = d2 / (d2 - d6);
        *wts = mk3(1.0f - t, 0.0f, t);
        return a + ac * t;
    }
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        *wts = mk3(0.0f, 1.0f - t, t);
        return b + (c - b) * t;
    }
    float denom = 1.0f / (va + vb + vc);
    float v = vb * denom, wv = vc * denom;
    *wts = mk3(1.0f - v - wv, v, wv);
    return a + ab * v + ac * wv;
}
__device__ __forceinline__ float face_span(f3 a, f3 b, f3 c) {
    return wmax(wmax(length(b - a), length(c - a)), length(c - b));
}
__device__ bool tetra_contains(const SPt* t) {
    const uint32_t faces[4][3] = {{0, 1, 2}, {0, 2, 3}, {0, 3, 1}, {1, 3, 2}};
    for (uint32_t f = 0; f < 4; ++f) {
        f3 a = t[faces[f][0]].w, b = t[faces[f][1]].w, c = t[faces[f][2]].w;
        f3 normal = cross(b - a, c - a);
        float span = face_span(a, b, c);
        if (length(normal) <= 1e-6f * span * span) return false;
        if (dot(normal, s3(0.0f) - a) > 0.0f) return false;
    }
    return true;
}
struct SRes {
    f3 v;
    float lam[4];
    bool pen;
    f3 pa, pb;
};
__device__ SRes simplex_closest(const SPt* s, uint32_t count) {
    SRes r;
    r.v = s3(3.402823466e38f);
    for (int i = 0; i < 4; ++i) r.lam[i] = 0.0f;
    r.pen = count == 4u && tetra_contains(s);
    r.pa = s3(0.0f);
    r.pb = s3(0.0f);
    if (r.pen) {
        r.v = s3(0.0f);
        return r;
    }
    for (uint32_t i = 0; i < count; ++i) {
        if (length(s[i].w) < length(r.v)) {
            r.v = s[i].w;
            for (int k = 0; k < 4; ++k) r.lam[k] = 0.0f;
            r.lam[i] = 1.0f;
        }
    }
    for (uint32_t i = 0; i < count; ++i) {
        for (uint32_t j = i + 1; j < count; ++j) {
            f3 a = s[i].w, b = s[j].w;
            f3 ab = b - a;
            float denom = dot(ab, ab);
            if (denom < 1e-12f) continue;
            float t = wclamp(-dot(a, ab) / denom, 0.0f, 1.0f);
            f3 point = a + ab * t;
            if (length(point) < length(r.v)) {
                r.v = point;
                for (int k = 0; k < 4; ++k) r.lam[k] = 0.0f;
                r.lam[i] = 1.0f - t;
                r.lam[j] = t;
            }
        }
    }
    if (count >= 3u) {
        for (uint32_t i = 0; i < count; ++i) {
            for (uint32_t j = i + 1; j < count; ++j) {
                for (uint32_t k = j + 1; k < count; ++k) {
                    f3 wts = s3(0.0f);
                    f3 point = closest_on_triangle(s[i].w, s[j].w, s[k].w, &wts);
                    if (length(point) < length(r.v)) {
                        r.v = point;
                        for (int q = 0; q < 4; ++q) r.lam[q] = 0.0f;
                        r.lam[i] = wts.x;
                        r.lam[j] = wts.y;
                        r.lam[k] = wts.z;
                    }
                }
            }
        }
    }
    for (uint32_t i = 0; i < count; ++i) {
        r.pa = r.pa + r.lam[i] * s[i].a;
        r.pb = r.pb + r.lam[i] * s[i].b;
    }
    return r;
}
__device__ __forceinline__ SPt support_pair(const DeviceWorld& w, const WShape& f, const WShape& s, f3 d) {
    f3 a = support(w, f, d);
    f3 b = support(w, s, -d);
    return SPt{a - b, a, b};
}
__device__ __forceinline__ float shape_scale(const WShape& s) {
    float scale = s.radius + s.half_height;
    scale = wmax(scale, wmax(wmax(s.half_extents.x, s.half_extents.y), s.half_extents.z));
    return wmax(scale, 1e-4f) * wmax(wmax(s.scale.x, s.scale.y), s.scale.z);
}
__device__ f3 simplex_expand_dir(const SPt* s, uint32_t count) {
    if (count == 1u) return mk3(1.0f, 0.0f, 0.0f);
    if (count == 2u) {
        f3 edge = s[1].w - s[0].w;
        f3 d = cross(edge, mk3(1.0f, 0.0f, 0.0f));
        if (length(d) < 1e-6f) d = cross(edge, mk3(0.0f, 1.0f, 0.0f));
        return normalize(d);
    }
    f3 normal = cross(s[1].w - s[0].w, s[2].w - s[0].w);
    if (length(normal) > 1e-8f) return normalize(normal);
    return mk3(0.0f, 1.0f, 0.0f);
}

struct Hit {
    float distance;
    f3 point, normal;
};

struct EpaOut {
    bool valid;
    f3 normal;
    float depth;
};

// convex.wgsl:286-437. The polytope lives in the calling thread's local memory.
__device__ EpaOut epa_tetrahedron(const DeviceWorld& w, const WShape& first, const WShape& second, const SPt* simplex) {
    f3 poly[64];
    uint8_t fa[128], fb[128], fcv[128];  // polytope indices are below 64
    f3 fn[128];
    uint8_t vis[128];
    uint8_t na[64], nb[64], nc[64];
    f3 nn[64];
    EpaOut invalid{false, mk3(0.0f, 1.0f, 0.0f), 0.0f};
    for (uint32_t i = 0; i < 4; ++i) poly[i] = simplex[i].w;
    uint32_t vc = 4;
    uint32_t fcount = 0;
    const uint32_t tet[4][3] = {{0, 1, 2}, {0, 2, 3}, {0, 3, 1}, {1, 3, 2}};
    for (uint32_t i = 0; i < 4; ++i) {
        uint32_t a = tet[i][0], b = tet[i][1], c = tet[i][2];
        f3 normal = cross(poly[b] - poly[a], poly[c] - poly[a]);
        float ln = length(normal);
        if (ln < 1e-10f) return invalid;
        f3 unit = normal / ln;
        f3 centroid = (poly[a] + poly[b] + poly[c]) * (1.0f / 3.0f);
        fa[fcount] = a;
        fb[fcount] = b;
        fcv[fcount] = c;
        fn[fcount] = dot(unit, centroid) > 0.0f ? -unit : unit;
        fcount += 1;
    }
    float best_dist = 0.0f;
    uint32_t best = 0;
    for (uint32_t iter = 0; iter < 32u; ++iter) {
        best_dist = 3.402823466e38f;
        best = 0;
        for (uint32_t i = 0; i < fcount; ++i) {
            float dist = dot(fn[i], poly[fa[i]]);
            if (dist < best_dist && length(fn[i]) > 0.5f) {
                best_dist = dist;
                best = i;
            }
        }
        f3 probe = support_pair(w, first, second, fn[best]).w;
        float gain = dot(probe, fn[best]) - best_dist;
        if (gain < 1e-4f) break;
        if (vc >= 64u) break;
        poly[vc] = probe;
        vc += 1;
        uint32_t vcount = 0;
        for (uint32_t i = 0; i < fcount; ++i) {
            if (dot(fn[i], probe - poly[fa[i]]) > 1e-6f) {
                vis[vcount] = i;
                vcount += 1;
            }
        }
        uint32_t ncount = 0;
        for (uint32_t i = 0; i < vcount; ++i) {
            uint32_t f = vis[i];
            uint32_t ea[3] = {fa[f], fb[f], fcv[f]};
            uint32_t eb[3] = {fb[f], fcv[f], fa[f]};
            for (uint32_t e = 0; e < 3; ++e) {
                uint32_t start = ea[e], end = eb[e];
                bool shared = false;
                for (uint32_t j = 0; j < vcount; ++j) {
                    if (j == i) continue;
                    uint32_t o = vis[j];
                    if ((fa[o] == end && fb[o] == start) || (fb[o] == end && fcv[o] == start) || (fcv[o] == end && fa[o] == start)) {
                        shared = true;
                    }
                }
                if (!shared && ncount < 64u) {
                    uint32_t apex = vc - 1u;
                    f3 normal = cross(poly[end] - poly[apex], poly[start] - poly[apex]);
                    float ln = length(normal);
                    if (ln > 1e-10f) {
                        f3 unit = normal / ln;
                        f3 centroid = (poly[apex] + poly[start] + poly[end]) * (1.0f / 3.0f);
                        na[ncount] = apex;
                        nb[ncount] = start;
                        nc[ncount] = end;
                        nn[ncount] = dot(unit, centroid) > 0.0f ? -unit : unit;
                        ncount += 1;
                    }
                }
            }
        }
        uint32_t write = 0, seen = 0;
        for (uint32_t i = 0; i < fcount; ++i) {
            if (seen < vcount && vis[seen] == i) {
                seen += 1;
                continue;
            }
            fa[write] = fa[i];
            fb[write] = fb[i];
            fcv[write] = fcv[i];
            fn[write] = fn[i];
            write += 1;
        }
        fcount = write;
        if (fcount + ncount > 128u) break;
        for (uint32_t i = 0; i < ncount; ++i) {
            fa[fcount] = na[i];
            fb[fcount] = nb[i];
            fcv[fcount] = nc[i];
            fn[fcount] = nn[i];
            fcount += 1;
        }
    }
    best_dist = 3.402823466e38f;
    for (uint32_t i = 0; i < fcount; ++i) {
        float dist = dot(fn[i], poly[fa[i]]);
        if (dist < best_dist && length(fn[i]) > 0.5f) {
            best_dist = dist;
            best = i;
        }
    }
    EpaOut r;
    r.valid = best_dist < 3.402823466e38f;
    r.normal = fn[best];
    r.depth = best_dist;
    return r;
}

__device__ __forceinline__ float support_projection_depth(const DeviceWorld& w, const WShape& f, const WShape& s, f3 direction) {
    f3 n = normalize(direction);
    return dot(support(w, f, n) - support(w, s, -n), n);
}
// convex.wgsl:532-582
// With stop_at_separation the probe returns as soon as one direction shows no overlap (depth <= 0):
// the caller then only needs to know that the minimum is not positive, and the minimum over all
// directions is unchanged whenever it is positive.
__device__ EpaOut penetration_probe(const DeviceWorld& w, const WShape& first, const WShape& second, const SPt* simplex,
                                    uint32_t count, bool stop_at_separation = false) {
    EpaOut best{false, mk3(0.0f, 1.0f, 0.0f), 3.402823466e38f};
    f3 probed[16];
    uint32_t pc = 0;
    for (uint32_t i = 0; i < count; ++i)
        for (uint32_t j = i + 1; j < count; ++j)
            for (uint32_t k = j + 1; k < count; ++k) {
                f3 normal = cross(simplex[j].w - simplex[i].w, simplex[k].w - simplex[i].w);
                if (length(normal) > 1e-8f && pc < 16u) probed[pc++] = normal;
            }
    f3 cdir = second.center - first.center;
    if (length(cdir) > 1e-8f && pc < 16u) probed[pc++] = cdir;
    const float ax[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (uint32_t i = 0; i < 6; ++i)
        if (pc < 16u) probed[pc++] = mk3(ax[i][0], ax[i][1], ax[i][2]);
    for (uint32_t i = 0; i < pc; ++i) {
        float depth = support_projection_depth(w, first, second, probed[i]);
        if (depth < best.depth) {
            best.depth = depth;
            best.normal = normalize(probed[i]);
        }
        if (stop_at_separation && depth <= 0.0f) break;
    }
    best.valid = best.depth < 3.402823466e38f;
    return best;
}

// convex.wgsl:464-521 then 584-618
__device__ Hit convex_hit(const DeviceWorld& w, const WShape& first, const WShape& second) {
    SPt s[4];
    uint32_t count = 0;
    float rdist = 0.0f;
    f3 rpa = first.center, rpb = second.center;
    f3 rnormal = sign_normalize(second.center - first.center);
    bool rpen = false;
    f3 dir = second.center - first.center;
    if (length(dir) < 1e-8f) dir = mk3(1.0f, 0.0f, 0.0f);
    s[0] = support_pair(w, first, second, dir);
    count = 1;
    SRes cl = simplex_closest(s, count);
    float tiny = 1e-4f * wmin(shape_scale(first), shape_scale(second));
    for (uint32_t iter = 0; iter < 24u; ++iter) {
        if (cl.pen || length(cl.v) < tiny) {
            while (count < 4u) {
                f3 d = simplex_expand_dir(s, count);
                s[count] = support_pair(w, first, second, d);
                count += 1;
            }
            rpen = true;
            rdist = 0.0f;
            rpa = cl.pa;
            rpb = cl.pb;
            break;
        }
        SPt sp = support_pair(w, first, second, -cl.v);
        if (dot(sp.w, -cl.v) <= dot(cl.v, -cl.v) + 1e-4f * wmax(1.0f, dot(cl.v, cl.v))) {
            rdist = length(cl.v);
            rpa = cl.pa;
            rpb = cl.pb;
            if (rdist > 1e-6f) rnormal = sign_normalize(cl.pb - cl.pa);
            break;
        }
        // simplex_reduce
        SPt kept[4];
        uint32_t kc = 0;
        for (uint32_t i = 0; i < 4; ++i) {
            if (cl.lam[i] > 1e-6f) kept[kc++] = s[i];
        }
        if (kc == 0u) {
            kept[0] = s[0];
            kc = 1;
        }
        for (uint32_t i = 0; i < kc; ++i) s[i] = kept[i];
        count = kc;
        // simplex_holds
        float span = shape_scale(second);
        float tol = (1e-5f * span) * (1e-5f * span);
        bool holds = false;
        for (uint32_t i = 0; i < count; ++i) {
            f3 off = s[i].w - sp.w;
            if (dot(off, off) <= tol) holds = true;
        }
        if (holds) {
            rdist = length(cl.v);
            rpa = cl.pa;
            rpb = cl.pb;
            if (rdist > 1e-6f) rnormal = sign_normalize(cl.pb - cl.pa);
            break;
        }
        s[count] = sp;
        count += 1;
        cl = simplex_closest(s, count);
    }
    if (!rpen) {
        EpaOut probe = penetration_probe(w, first, second, s, count, true);
        if (probe.depth > 0.0f) {
            f3 normal = probe.normal;
            if (dot(normal, second.center - first.center) < 0.0f) normal = -normal;
            return Hit{-probe.depth, (rpa + rpb) * 0.5f, normal};
        }
        if (rdist > 0.0f) return Hit{rdist, (rpa + rpb) * 0.5f, rnormal};
        return Hit{3.402823466e38f, s3(0.0f), s3(0.0f)};
    }
    EpaOut epa = epa_tetrahedron(w, first, second, s);
    Hit result;
    if (epa.valid && epa.depth > 0.0f && epa.depth < 3.402823466e38f && length(epa.normal) > 0.5f
        && epa.depth < support_projection_depth(w, first, second, epa.normal) + 0.1f * wmin(shape_scale(first), shape_scale(second))) {
        f3 pa = support(w, first, epa.normal);
        f3 pb = support(w, second, -epa.normal);
        result = Hit{-epa.depth, (pa + pb) * 0.5f, epa.normal};
    } else {
        EpaOut probe = penetration_probe(w, first, second, s, count);
        f3 pa = support(w, first, probe.normal);
        f3 pb = support(w, second, -probe.normal);
        result = Hit{-probe.depth, (pa + pb) * 0.5f, probe.normal};
    }
    if (dot(result.normal, second.center - first.center) < 0.0f) result.normal = -result.normal;
    return result;
}

// ---- the convex path in three phases (results identical to convex_hit) ----
//
// Phase 1, one thread per pair: GJK (convex.wgsl:464-521) and, for separated shapes, the
// penetration probe that may still report overlap (convex.wgsl:588-600). Phase 2, one warp per
// penetrating pair: EPA (convex.wgsl:286-437) with the polytope in shared memory and its face
// loops spread over the lanes, then the acceptance test and probe fallback (convex.wgsl:602-617).
// Phase 3, one thread per hit: the feature-ring manifold.

struct GjkOut {
    bool pen;
    bool rejected;  // the centre-axis gap already exceeds the caller's margin: no contact
    uint32_t count;
    float dist;
    f3 pa, pb, normal;
    SPt s[4];
};

// With reject_gap > 0, a pair whose gap along the centre axis exceeds reject_gap returns at once
// with `rejected` set. That answer equals the full path's: the first support point is taken along
// that axis, a gap g along any unit axis bounds the true distance from below, GJK's reported
// distance (the closest point of a simplex inside the Minkowski difference) is at least the true
// distance, and the penetration probe includes the centre axis, whose depth is -g < 0. So the full
// path reports either a distance >= g or no hit, and the caller discards both when g exceeds its
// margin; reject_gap carries a tolerance above the margin for the rounding of the dot products.
__device__ GjkOut gjk_phase(const DeviceWorld& w, const WShape& first, const WShape& second, float reject_gap = -1.0f) {
    GjkOut o;
    o.rejected = false;
    o.count = 0;
    o.dist = 0.0f;
    o.pa = first.center;
    o.pb = second.center;
    o.normal = sign_normalize(second.center - first.center);
    o.pen = false;
    f3 dir = second.center - first.center;
    if (length(dir) < 1e-8f) dir = mk3(1.0f, 0.0f, 0.0f);
    o.s[0] = support_pair(w, first, second, dir);
    o.count = 1;
    if (reject_gap > 0.0f && dot(o.s[0].w, dir) < -reject_gap * length(dir)) {
        o.rejected = true;
        return o;
    }
    SRes cl = simplex_closest(o.s, o.count);
    float tiny = 1e-4f * wmin(shape_scale(first), shape_scale(second));
    for (uint32_t iter = 0; iter < 24u; ++iter) {
        if (cl.pen || length(cl.v) < tiny) {
            while (o.count < 4u) {
                f3 d = simplex_expand_dir(o.s, o.count);
                o.s[o.count] = support_pair(w, first, second, d);
                o.count += 1;
            }
            o.pen = true;
            o.dist = 0.0f;
            o.pa = cl.pa;
            o.pb = cl.pb;
            break;
        }
        SPt sp = support_pair(w, first, second, -cl.v);
        if (dot(sp.w, -cl.v) <= dot(cl.v, -cl.v) + 1e-4f * wmax(1.0f, dot(cl.v, cl.v))) {
            o.dist = length(cl.v);
            o.pa = cl.pa;
            o.pb = cl.pb;
            if (o.dist > 1e-6f) o.normal = sign_normalize(cl.pb - cl.pa);
            break;
        }
        SPt kept[4];
        uint32_t kc = 0;
        for (uint32_t i = 0; i < 4; ++i) {
            if (cl.lam[i] > 1e-6f) kept[kc++] = o.s[i];
        }
        if (kc == 0u) {
            kept[0] = o.s[0];
            kc = 1;
        }
        for (uint32_t i = 0; i < kc; ++i) o.s[i] = kept[i];
        o.count = kc;
        float span = shape_scale(second);
        float tol = (1e-5f * span) * (1e-5f * span);
        bool holds = false;
        for (uint32_t i = 0; i < o.count; ++i) {
            f3 off = o.s[i].w - sp.w;
            if (dot(off, off) <= tol) holds = true;
        }
        if (holds) {
            o.dist = length(cl.v);
            o.pa = cl.pa;
            o.pb = cl.pb;
            if (o.dist > 1e-6f) o.normal = sign_normalize(cl.pb - cl.pa);
            break;
        }
        o.s[o.count] = sp;
        o.count += 1;
        cl = simplex_closest(o.s, o.count);
    }
    return o;
}

// convex.wgsl:588-600 for a separated GJK result.
__device__ Hit separated_hit(const DeviceWorld& w, const WShape& first, const WShape& second, const GjkOut& g) {
    EpaOut probe = penetration_probe(w, first, second, g.s, g.count, true);
    if (probe.depth > 0.0f) {
        f3 normal = probe.normal;
        if (dot(normal, second.center - first.center) < 0.0f) normal = -normal;
        return Hit{-probe.depth, (g.pa + g.pb) * 0.5f, normal};
    }
    if (g.dist > 0.0f) return Hit{g.dist, (g.pa + g.pb) * 0.5f, g.normal};
    return Hit{3.402823466e38f, s3(0.0f), s3(0.0f)};
}

// ---- warp-cooperative pieces ----
constexpr uint32_t kFull = 0xFFFFFFFFu;

// A group of G consecutive lanes of a warp (G = 32: the whole warp) working on one pair: its lane
// numbers, its member mask, and the warp intrinsics restricted to it.
template <uint32_t G>
struct Lanes {
    static_assert(G == 32u || G == 16u || G == 8u, "a lane group is a power-of-two part of a warp");
    uint32_t lane, base, mask;
    __device__ __forceinline__ Lanes() {
        const uint32_t l = threadIdx.x & 31u;
        lane = l & (G - 1u);
        base = l - lane;
        if constexpr (G == 32u) {
            mask = kFull;
        } else {
            mask = ((1u << G) - 1u) << base;
        }
    }
    __device__ __forceinline__ uint32_t ballot(bool p) const {
        const uint32_t b = __ballot_sync(mask, p) >> base;
        if constexpr (G == 32u) {
            return b;
        } else {
            return b & ((1u << G) - 1u);
        }
    }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    __device__ __forceinline__ bool any(bool p) const { return __any_sync(mask, p); }
    __device__ __forceinline__ uint32_t max(uint32_t v) const { return __reduce_max_sync(mask, v); }
    __device__ __forceinline__ uint32_t min(uint32_t v) const { return __reduce_min_sync(mask, v); }
    template <class T>
    __device__ __forceinline__ T shfl(T v, uint32_t src) const { return __shfl_sync(mask, v, (int)src, (int)G); }
};

// An unsigned key that orders floats above -FLT_MAX as the floats compare: -0 and +0 share a key
// (they compare equal), and NaN, -inf and -FLT_MAX (never above the scans' -FLT_MAX start) get 0.
__device__ __forceinline__ uint32_t order_key(float x) {
    if (!(x > -3.402823466e38f)) return 0u;
    const uint32_t b = __float_as_uint(x == 0.0f ? 0.0f : x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
// The first maximum of a group-wide scan: the largest key, then the lowest index among the lanes
// that hold it (each lane holds the first index of its own maximum). Returns 0xFFFFFFFF when no
// lane holds a candidate.
template <uint32_t G>
__device__ __forceinline__ uint32_t warp_first_max(const Lanes<G>& L, uint32_t key, uint32_t index) {
    const uint32_t top = L.max(key);
    if (top == 0u) return 0xFFFFFFFFu;
    return L.min(key == top ? index : 0xFFFFFFFFu);
}

// support_local over a hull with the warp's lanes striding the vertices; the reduction keeps the
// sequential scan's choice: the largest dot product, the lowest index among equal ones.
template <uint32_t G>
__device__ __forceinline__ f3 warp_support_local(const Lanes<G>& L, const DeviceWorld& w, const WShape& s, f3 d) {
    if (s.kind != 5u) return support_local(w, s, d);
    const dyn_shape_source_record& src = w.sources[s.source];
    const float4* verts = w.vertices + src.vertex_offset;
    float best = -3.402823466e38f;
    uint32_t bi = 0xFFFFFFFFu;
    for (uint32_t i = L.lane; i < src.vertex_count; i += G) {
        float sd = dot(xyz(__ldg(verts + i)), d);
        if (sd > best) {
            best = sd;
            bi = i;
        }
    }
    bi = warp_first_max(L, bi == 0xFFFFFFFFu ? 0u : order_key(best), bi);
    return bi == 0xFFFFFFFFu ? s3(0.0f) : xyz(__ldg(verts + bi));
}
template <uint32_t G>
__device__ __forceinline__ f3 warp_support(const Lanes<G>& L, const DeviceWorld& w, const WShape& s, f3 direction) {
    f3 local_d = quat_rotate(quat_conj(s.rotation), direction);
    f3 local = warp_support_local(L, w, s, local_d * s.scale);
    return s.center + quat_rotate(s.rotation, local * s.scale);
}

struct EpaWarpShared {
    float4 poly[64];
    float4 fn[128];      // face normal.xyz, packed (a | b << 8 | c << 16) bits in w
    float4 nn[64];
    uint8_t vis[128];
    uint8_t visflag[128];
};

__device__ __forceinline__ float4 pack_face(f3 n, uint32_t a, uint32_t b, uint32_t c) {
    return make_float4(n.x, n.y, n.z, __uint_as_float(a | (b << 8) | (c << 16)));
}
__device__ __forceinline__ void unpack_face(float4 f, uint32_t* a, uint32_t* b, uint32_t* c) {
    uint32_t bits = __float_as_uint(f.w);
    *a = bits & 255u;
    *b = (bits >> 8) & 255u;
    *c = (bits >> 16) & 255u;
}

// (min distance, lowest index) over faces whose normal is longer than 0.5: the first minimum of
// convex.wgsl:344-352, identical on every lane.
template <uint32_t G>
__device__ __forceinline__ void warp_best_face(const Lanes<G>& L, const EpaWarpShared& m, uint32_t fcount, float* best_dist,
                                               uint32_t* best_face) {
    float bd = 3.402823466e38f;
    uint32_t bi = 0u;
    bool any = false;
    for (uint32_t j = L.lane; j < fcount; j += G) {
        float4 f = m.fn[j];
        uint32_t a, b, c;
        unpack_face(f, &a, &b, &c);
        f3 n = xyz(f);
        float dist = dot(n, xyz(m.poly[a]));
        if (dist < bd && length(n) > 0.5f) {
            bd = dist;
            bi = j;
            any = true;
        }
    }
    // the first minimum: the first maximum of the negated distances (negation is exact)
    const uint32_t first = warp_first_max(L, any ? order_key(-bd) : 0u, any ? bi : 0xFFFFFFFFu);
    if (first == 0xFFFFFFFFu) {
        *best_dist = 3.402823466e38f;
        *best_face = 0u;
        return;
    }
    *best_dist = L.shfl(bd, first & (G - 1u));  // face j lives on lane j % G
    *best_face = first;
}

// convex.wgsl:286-437 on one warp. All lanes return the same result.
template <uint32_t G>
__device__ EpaOut warp_epa(const Lanes<G>& L, const DeviceWorld& w, const WShape& first, const WShape& second,
                           const f3* simplex, EpaWarpShared& m) {
    const uint32_t lane = L.lane;
    const uint32_t lt = (1u << lane) - 1u;
    EpaOut invalid{false, mk3(0.0f, 1.0f, 0.0f), 0.0f};
    if (lane < 4u) m.poly[lane] = mk4(simplex[lane], 0.0f);
    L.sync();
    const uint32_t tet[4][3] = {{0, 1, 2}, {0, 2, 3}, {0, 3, 1}, {1, 3, 2}};
    bool bad = false;
    if (lane < 4u) {
        uint32_t a = tet[lane][0], b = tet[lane][1], c = tet[lane][2];
        f3 pa = xyz(m.poly[a]), pb = xyz(m.poly[b]), pc = xyz(m.poly[c]);
        f3 normal = cross(pb - pa, pc - pa);
        float ln = length(normal);
        if (ln < 1e-10f) {
            bad = true;
        } else {
            f3 unit = normal / ln;
            f3 centroid = (pa + pb + pc) * (1.0f / 3.0f);
            m.fn[lane] = pack_face(dot(unit, centroid) > 0.0f ? -unit : unit, a, b, c);
        }
    }
    if (L.any(bad)) return invalid;
    L.sync();
    uint32_t fcount = 4, vc = 4;
    float bd = 0.0f;
    uint32_t bf = 0;
    for (uint32_t iter = 0; iter < 32u; ++iter) {
        warp_best_face(L, m, fcount, &bd, &bf);
        f3 n = xyz(m.fn[bf]);
        f3 probe = warp_support(L, w, first, n) - warp_support(L, w, second, -n);
        float gain = dot(probe, n) - bd;
        if (gain < 1e-4f) break;
        if (vc >= 64u) break;
        L.sync();
        if (lane == 0u) m.poly[vc] = mk4(probe, 0.0f);
        vc += 1;
        // visible faces in index order
        uint32_t vcount = 0;
        for (uint32_t base = 0; base < fcount; base += G) {
            uint32_t j = base + lane;
            bool v = false;
            if (j < fcount) {
                float4 f = m.fn[j];
                uint32_t a, b, c;
                unpack_face(f, &a, &b, &c);
                v = dot(xyz(f), probe - xyz(m.poly[a])) > 1e-6f;
                m.visflag[j] = v ? 1u : 0u;
            }
            uint32_t mask = L.ballot(v);
            if (v) m.vis[vcount + __popc(mask & lt)] = (uint8_t)j;
            vcount += __popc(mask);
        }
        L.sync();
        // horizon edges become new faces, in (visible face, edge) order, at most 64
        uint32_t ncount = 0;
        const uint32_t apex = vc - 1u;
        for (uint32_t base = 0; base < 3u * vcount; base += G) {
            uint32_t t = base + lane;
            bool keep = false;
            float4 face = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (t < 3u * vcount) {
                uint32_t i = t / 3u, e = t % 3u;
                uint32_t a, b, c;
                unpack_face(m.fn[m.vis[i]], &a, &b, &c);
                uint32_t start = e == 0u ? a : (e == 1u ? b : c);
                uint32_t end = e == 0u ? b : (e == 1u ? c : a);
                bool shared = false;
                for (uint32_t jj = 0; jj < vcount; ++jj) {
                    if (jj == i) continue;
                    uint32_t oa, ob, oc;
                    unpack_face(m.fn[m.vis[jj]], &oa, &ob, &oc);
                    if ((oa == end && ob == start) || (ob == end && oc == start) || (oc == end && oa == start)) shared = true;
                }
                if (!shared) {
                    f3 pap = xyz(m.poly[apex]), ps = xyz(m.poly[start]), pe = xyz(m.poly[end]);
                    f3 normal = cross(pe - pap, ps - pap);
                    float ln = length(normal);
                    if (ln > 1e-10f) {
                        f3 unit = normal / ln;
                        f3 centroid = (pap + ps + pe) * (1.0f / 3.0f);
                        face = pack_face(dot(unit, centroid) > 0.0f ? -unit : unit, apex, start, end);
                        keep = true;
                    }
                }
            }
            uint32_t mask = L.ballot(keep);
            uint32_t rank = ncount + __popc(mask & lt);
            if (keep && rank < 64u) m.nn[rank] = face;
            ncount = min(ncount + (uint32_t)__popc(mask), 64u);
        }
        L.sync();
        // drop the visible faces, keeping order
        uint32_t write = 0;
        for (uint32_t base = 0; base < fcount; base += G) {
            uint32_t j = base + lane;
            bool keepf = j < fcount && m.visflag[j] == 0u;
            float4 f = j < fcount ? m.fn[j] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            uint32_t mask = L.ballot(keepf);
            L.sync();
            if (keepf) m.fn[write + __popc(mask & lt)] = f;
            write += __popc(mask);
            L.sync();
        }
        fcount = write;
        if (fcount + ncount > 128u) break;
        for (uint32_t t = lane; t < ncount; t += G) m.fn[fcount + t] = m.nn[t];
        fcount += ncount;
        L.sync();
    }
    L.sync();
    float fd = 3.402823466e38f;
    uint32_t ff = bf;
    {
        float d2;
        uint32_t f2;
        warp_best_face(L, m, fcount, &d2, &f2);
        fd = d2;
        if (d2 < 3.402823466e38f) ff = f2;
    }
    EpaOut r;
    r.valid = fd < 3.402823466e38f;
    r.normal = xyz(m.fn[ff < 128u ? ff : 0u]);
    r.depth = fd;
    return r;
}

template <uint32_t G>
__device__ __forceinline__ float warp_projection_depth(const Lanes<G>& L, const DeviceWorld& w, const WShape& f, const WShape& s,
                                                       f3 direction) {
    f3 n = normalize(direction);
    return dot(warp_support(L, w, f, n) - warp_support(L, w, s, -n), n);
}

// convex.wgsl:602-617 after a penetrating GJK (one warp, every lane returns the same hit).
template <uint32_t G>
__device__ Hit warp_penetrating_hit(const Lanes<G>& L, const DeviceWorld& w, const WShape& first, const WShape& second,
                                    const f3* simplex, EpaWarpShared& m) {
    EpaOut epa = warp_epa(L, w, first, second, simplex, m);
    Hit result;
    bool accept = epa.valid && epa.depth > 0.0f && epa.depth < 3.402823466e38f && length(epa.normal) > 0.5f;
    if (accept) {
        accept = epa.depth < warp_projection_depth(L, w, first, second, epa.normal) + 0.1f * wmin(shape_scale(first), shape_scale(second));
    }
    if (accept) {
        f3 pa = warp_support(L, w, first, epa.normal);
        f3 pb = warp_support(L, w, second, -epa.normal);
        result = Hit{-epa.depth, (pa + pb) * 0.5f, epa.normal};
    } else {
        // convex_penetration_probe over the four-point simplex, centre direction and six axes: each
        // direction's projection depth on its own lane (the lane scans the vertices itself), then
        // the first minimum in direction order, as the sequential loop keeps it
        f3 probed[16];
        uint32_t pc = 0;
        for (uint32_t i = 0; i < 4; ++i)
            for (uint32_t j = i + 1; j < 4; ++j)
                for (uint32_t k = j + 1; k < 4; ++k) {
                    f3 normal = cross(simplex[j] - simplex[i], simplex[k] - simplex[i]);
                    if (length(normal) > 1e-8f && pc < 16u) probed[pc++] = normal;
                }
        f3 cdir = second.center - first.center;
        if (length(cdir) > 1e-8f && pc < 16u) probed[pc++] = cdir;
        const float ax[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        for (uint32_t i = 0; i < 6; ++i)
            if (pc < 16u) probed[pc++] = mk3(ax[i][0], ax[i][1], ax[i][2]);
        const uint32_t lane = L.lane;  // pc <= 11 < G: one direction per lane
        const float mine = lane < pc ? support_projection_depth(w, first, second, probed[lane]) : 3.402823466e38f;
        float best_depth = 3.402823466e38f;
        uint32_t best_i = pc;
        for (uint32_t i = 0; i < pc; ++i) {
            const float depth = L.shfl(mine, i);
            if (depth < best_depth) {
                best_depth = depth;
                best_i = i;
            }
        }
        const f3 best_normal = best_i < pc ? normalize(probed[best_i]) : mk3(0.0f, 1.0f, 0.0f);
        f3 pa = warp_support(L, w, first, best_normal);
        f3 pb = warp_support(L, w, second, -best_normal);
        result = Hit{-best_depth, (pa + pb) * 0.5f, best_normal};
    }
    if (dot(result.normal, second.center - first.center) < 0.0f) result.normal = -result.normal;
    return result;
}

// ---- features (convex.wgsl:639-900) ----
__device__ uint32_t box_feature_ring(const WShape& s, f3 direction, f3* out, uint32_t* ids, uint32_t* face) {
    f3 axes[3] = {quat_rotate(s.rotation, mk3(1.0f, 0.0f, 0.0f)), quat_rotate(s.rotation, mk3(0.0f, 1.0f, 0.0f)),
                  quat_rotate(s.rotation, mk3(0.0f, 0.0f, 1.0f))};
    uint32_t best = 0;
    for (uint32_t i = 1; i < 3; ++i) {
        if (fabsf(dot(axes[i], direction)) > fabsf(dot(axes[best], direction))) best = i;
    }
    float sign = dot(axes[best], direction) < 0.0f ? -1.0f : 1.0f;
    f3 fdir = axes[best] * sign;
    f3 center = s.center + fdir * comp(s.half_extents, best);
    f3 u1 = axes[(best + 1u) % 3u], u2 = axes[(best + 2u) % 3u];
    float e1 = comp(s.half_extents, (best + 1u) % 3u), e2 = comp(s.half_extents, (best + 2u) % 3u);
    out[0] = center + u1 * e1 + u2 * e2;
    ids[0] = box_corner_id(best, sign, 1.0f, 1.0f);
    out[1] = center - u1 * e1 + u2 * e2;
    ids[1] = box_corner_id(best, sign, -1.0f, 1.0f);
    out[2] = center - u1 * e1 - u2 * e2;
    ids[2] = box_corner_id(best, sign, -1.0f, -1.0f);
    out[3] = center + u1 * e1 - u2 * e2;
    ids[3] = box_corner_id(best, sign, 1.0f, -1.0f);
    *face = kFeatFaceBit | (best * 2u + (sign > 0.0f ? 1u : 0u));
    return 4;
}
__device__ uint32_t ring_of(const DeviceWorld& w, const WShape& s, f3 direction, f3* pts, uint32_t* ids, uint32_t count,
                            f3* out, uint32_t* out_ids) {
    if (count <= 1u) {
        out[0] = support(w, s, direction);
        out_ids[0] = ids[0];
        return 1;
    }
    f3 n = sign_normalize(direction);
    f3 center = s3(0.0f);
    for (uint32_t i = 0; i < count; ++i) center = center + pts[i];
    center = center / (float)count;
    f3 u = fabsf(n.x) > 0.9f ? normalize(cross(n, mk3(0.0f, 1.0f, 0.0f))) : normalize(cross(n, mk3(1.0f, 0.0f, 0.0f)));
    f3 v = cross(n, u);
    // convex.wgsl:699-714 compares atan2 angles of the points currently at i and j; a point's
    // angle does not depend on where it sits, so each is computed once and travels with it.
    float angle[16];
    for (uint32_t i = 0; i < count; ++i) {
        f3 pa = pts[i] - center;
        angle[i] = datan2(dot(pa, v), dot(pa, u));
    }
    for (uint32_t i = 0; i < count; ++i) {
        for (uint32_t j = i + 1; j < count; ++j) {
            if (angle[j] < angle[i]) {
                f3 t = pts[i];
                pts[i] = pts[j];
                pts[j] = t;
                uint32_t ti = ids[i];
                ids[i] = ids[j];
                ids[j] = ti;
                float ta = angle[i];
                angle[i] = angle[j];
                angle[j] = ta;
            }
        }
    }
    uint32_t keep = count < 8u ? count : 8u;
    for (uint32_t i = 0; i < keep; ++i) {
        out[i] = pts[i];
        out_ids[i] = ids[i];
    }
    return keep;
}
__device__ uint32_t hull_feature_ring(const DeviceWorld& w, const WShape& s, f3 direction, f3* out, uint32_t* ids, uint32_t* face) {
    const dyn_shape_source_record& src = w.sources[s.source];
    f3 d = quat_rotate(quat_conj(s.rotation), direction) * s.scale;
    float best_dot = dot(support_local(w, s, d), d);
    f3 extent = mk3(src.local_max[0], src.local_max[1], src.local_max[2]) - mk3(src.local_min[0], src.local_min[1], src.local_min[2]);
    float eps = 1e-3f * wmax(wmax(extent.x, extent.y), extent.z) * wmax(wmax(s.scale.x, s.scale.y), s.scale.z);
    f3 pts[16];
    uint32_t pid[16];
    uint32_t count = 0;
    uint32_t first_id = 1u << 12;
    const float4* verts = w.vertices + src.vertex_offset;
    for (uint32_t i = 0; i < src.vertex_count && count < 16u; ++i) {
        f3 v = xyz(__ldg(verts + i));
        if (dot(v, d) >= best_dot - eps) {
            pts[count] = s.center + quat_rotate(s.rotation, v * s.scale);
            pid[count] = i;
            first_id = first_id < i ? first_id : i;
            count += 1;
        }
    }
    *face = kFeatFaceBit | first_id;
    return ring_of(w, s, direction, pts, pid, count, out, ids);
}
__device__ uint32_t shape_feature(const DeviceWorld& w, const WShape& s, f3 direction, f3* out, uint32_t* ids, uint32_t* face,
                                  bool* ring) {
    if (s.kind == 2u) {
        *ring = true;
        return box_feature_ring(s, direction, out, ids, face);
    }
    if (s.kind == 5u) {
        uint32_t c = hull_feature_ring(w, s, direction, out, ids, face);
        *ring = c > 2u;
        return c;
    }
    if (s.kind == 3u) {
        // capsule_feature (convex.wgsl:795-819)
        *ring = false;
        f3 ld = quat_rotate(quat_conj(s.rotation), direction) * s.scale;
        float cap = ld.y > 0.0f ? 1.0f : -1.0f;
        f3 radial = sign_normalize(ld) * s.radius;
        *face = kFeatFaceBit;
        if (fabsf(ld.y) > 0.93f * length(ld)) {
            f3 local = mk3(0.0f, cap * s.half_height, 0.0f) + radial;
            out[0] = s.center + quat_rotate(s.rotation, local * s.scale);
            ids[0] = cap > 0.0f ? 1u : 0u;
            return 1;
        }
        f3 upper = mk3(0.0f, s.half_height, 0.0f) + radial;
        f3 lower = mk3(0.0f, -s.half_height, 0.0f) + radial;
        out[0] = s.center + quat_rotate(s.rotation, upper * s.scale);
        out[1] = s.center + quat_rotate(s.rotation, lower * s.scale);
        ids[0] = 0;
        ids[1] = 1;
        return 2;
    }
    if (s.kind == 4u) {
        // cylinder_feature (convex.wgsl:821-854)
        f3 axis = quat_rotate(s.rotation, mk3(0.0f, 1.0f, 0.0f));
        float alignment = dot(axis, normalize(direction));
        if (fabsf(alignment) > 0.93f) {
            float sign = alignment < 0.0f ? -1.0f : 1.0f;
            uint32_t cap = sign > 0.0f ? 1u : 0u;
            f3 cc = s.center + axis * s.half_height * sign;
            f3 u = normalize(cross(axis, mk3(1.0f, 0.0f, 0.0f)));
            if (length(cross(axis, mk3(1.0f, 0.0f, 0.0f))) < 1e-6f) u = normalize(cross(axis, mk3(0.0f, 0.0f, 1.0f)));
            f3 v = cross(axis, u);
            for (uint32_t i = 0; i < 8u; ++i) {
                float angle = (float)i * 0.78539816f;
                out[i] = cc + (u * dcos(angle) + v * dsin(angle)) * s.radius;
                ids[i] = cap * 8u + i;
            }
            *face = kFeatFaceBit | cap;
            *ring = true;
            return 8;
        }
        f3 side = sign_normalize(direction - axis * dot(direction, axis));
        out[0] = s.center + axis * s.half_height + side * s.radius;
        ids[0] = 16u;
        out[1] = s.center - axis * s.half_height + side * s.radius;
        ids[1] = 17u;
        *face = kFeatFaceBit | 2u;
        *ring = false;
        return 2;
    }
    *ring = false;
    out[0] = support(w, s, direction);
    ids[0] = 0;
    *face = kFeatFaceBit;
    return 1;
}
__device__ __forceinline__ float feature_radius(const f3* p, uint32_t count) {
    f3 center = s3(0.0f);
    for (uint32_t i = 0; i < count; ++i) center = center + p[i];
    center = center / (float)count;
    float r = 0.0f;
    for (uint32_t i = 0; i < count; ++i) r = wmax(r, length(p[i] - center));
    return r;
}
// convex.wgsl:910-982
__device__ uint32_t clip_feature_to_ring(const f3* pts, const uint32_t* ids, uint32_t count, const f3* ring, uint32_t rc,
                                         f3 ref_dir, f3* held, uint32_t* hid) {
    for (uint32_t i = 0; i < count; ++i) {
        held[i] = pts[i];
        hid[i] = ids[i];
    }
    uint32_t live = count;
    for (uint32_t side = 0; side < rc; ++side) {
        f3 cur = ring[side];
        f3 nxt = ring[(side + 1u) % rc];
        f3 pn = normalize(cross(nxt - cur, ref_dir));
        f3 kp[16];
        uint32_t ki[16];
        uint32_t written = 0;
        if (live == 2u) {
            f3 p0 = held[0], p1 = held[1];
            float s0 = dot(p0 - cur, pn) - kClipMargin;
            float s1 = dot(p1 - cur, pn) - kClipMargin;
            if (s0 <= 0.0f) {
                kp[written] = p0;
                ki[written] = hid[0];
                written += 1;
            }
            if (s0 * s1 < 0.0f && written < 16u) {
                kp[written] = p0 + (p1 - p0) * (s0 / (s0 - s1));
                ki[written] = kFeatClip | (side * 16u);
                written += 1;
            }
            if (s1 <= 0.0f && written < 16u) {
                kp[written] = p1;
                ki[written] = hid[1];
                written += 1;
            }
        } else {
            for (uint32_t i = 0; i < live; ++i) {
                f3 cp = held[i];
                f3 np = held[(i + 1u) % live];
                float cs = dot(cp - cur, pn) - kClipMargin;
                float ns = dot(np - cur, pn) - kClipMargin;
                if (cs <= 0.0f && written < 16u) {
                    kp[written] = cp;
                    ki[written] = hid[i];
                    written += 1;
                }
                if (cs * ns < 0.0f && written < 16u) {
                    kp[written] = cp + (np - cp) * (cs / (cs - ns));
                    ki[written] = kFeatClip | (side * 16u + i);
                    written += 1;
                }
            }
        }
        live = written;
        for (uint32_t i = 0; i < written; ++i) {
            held[i] = kp[i];
            hid[i] = ki[i];
        }
        if (live == 0u) break;
    }
    return live;
}
// convex.wgsl:984-1071
__device__ bool convex_pair_manifold(const DeviceWorld& w, const WShape& first, const WShape& second, f3 direction, Mani* m) {
    f3 fp[8], sp[8];
    uint32_t fi[8], si[8];
    uint32_t ff = 0, sf = 0;
    bool fr = false, sr = false;
    uint32_t fcn = shape_feature(w, first, direction, fp, fi, &ff, &fr);
    uint32_t scn = shape_feature(w, second, -direction, sp, si, &sf, &sr);
    if (!fr && !sr) return false;
    bool first_ref = fr;
    if (fr && sr) first_ref = feature_radius(fp, fcn) >= feature_radius(sp, scn);
    const f3* ref = first_ref ? fp : sp;
    uint32_t rc = first_ref ? fcn : scn;
    uint32_t ref_face = first_ref ? ff : sf;
    const f3* inc = first_ref ? sp : fp;
    const uint32_t* inc_ids = first_ref ? si : fi;
    uint32_t ic = first_ref ? scn : fcn;
    f3 ref_dir = first_ref ? direction : -direction;
    f3 center = s3(0.0f);
    for (uint32_t i = 0; i < rc; ++i) center = center + ref[i];
    center = center / (float)rc;
    f3 deepest = s3(0.0f);
    float deepest_depth = -1e30f;
    for (uint32_t i = 0; i < ic; ++i) {
        float depth = dot(center - inc[i], ref_dir);
        if (depth > deepest_depth) {
            deepest_depth = depth;
            deepest = inc[i];
        }
    }
    f3 cp[16];
    uint32_t cid[16];
    uint32_t clipped = clip_feature_to_ring(inc, inc_ids, ic, ref, rc, ref_dir, cp, cid);
    Cand cands[16];
    uint32_t cc = 0;
    for (uint32_t i = 0; i < clipped && cc < 16u; ++i) {
        float depth = dot(center - cp[i], ref_dir);
        if (depth > 0.0f) {
            cands[cc] = Cand{cp[i] - ref_dir * (depth * 0.5f), depth,
                             first_ref ? feature_pair(kFeatVertex, ref_face, cid[i]) : feature_pair(kFeatVertex, cid[i], ref_face)};
            cc += 1;
        }
    }
    if (cc == 0u) {
        if (deepest_depth <= 0.0f) return false;
        mani_push(m, deepest - ref_dir * (deepest_depth * 0.5f), deepest_depth, kFeatPoint);
        return true;
    }
    mani_keep(m, cands, cc);
    return true;
}
// narrowphase.wgsl:485-512
// Slack below -margin before a plane pair is answered from the convex's deepest point alone: far
// above the rounding of the feature points at world coordinates of a few hundred metres.
constexpr float kPlaneRejectTolerance = 1e-3f;
__device__ Mani plane_convex(const DeviceWorld& w, const WShape& plane, const WShape& convex, float margin) {
    Mani m;
    f3 n = quat_rotate(plane.rotation, mk3(0.0f, 1.0f, 0.0f));
    float side = dot(convex.center - plane.center, n);
    f3 facing = side < 0.0f ? -n : n;
    mani_emit(&m, facing);
    // Every feature point below is a point of the convex, so none is deeper than its support point
    // along -facing: when that one is clear of the margin by more than rounding, no point is kept.
    if (dot(plane.center - support(w, convex, -facing), facing) < -(margin + kPlaneRejectTolerance)) return m;
    f3 pts[8];
    uint32_t ids[8];
    uint32_t feature = 0;
    bool ring = false;
    uint32_t count = shape_feature(w, convex, -facing, pts, ids, &feature, &ring);
    Cand cands[16];
    uint32_t cc = 0;
    for (uint32_t i = 0; i < count; ++i) {
        float depth = dot(plane.center - pts[i], facing);
        if (depth <= -margin) continue;
        cands[cc] = Cand{pts[i] + facing * (depth * 0.5f), depth, feature_pair(kFeatVertex, kFeatFaceBit, ids[i])};
        cc += 1;
    }
    mani_keep(&m, cands, cc);
    return m;
}

}  // namespace dyn
