// scene.cpp - host-side scene building of the C ABI: configuration, hulls, spawning, records.
//
// Restates the reference's host set-up for the step path:
//   PhysicsConfig::default                 crates/dynamis-model/src/config.rs:76-100
//   BodyStateRecord::initial               crates/dynamis-abi/src/body.rs:36-58
//   BodyDescriptorRecord::build            crates/dynamis-abi/src/body.rs:96-140
//   ColliderRecord::build                  crates/dynamis-abi/src/collider.rs:47-103
//   compute_mass_properties                crates/dynamis-model/src/mass.rs:155-212
//   hull solid integrals                   crates/dynamis-hull/src/solid.rs:62-105
//   StepParamsRecord::new                  crates/dynamis-abi/src/param.rs:110-158
//   hull (add_hull_from_mesh)              crates/dynamis-hull/src/hull.rs:53-288
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>

#include "world.h"

namespace dyn {

dyn_status fail(dyn_world* w, dyn_status status, const std::string& what) {
    if (w) w->last_error = what;
    return status;
}

namespace {

using D3 = std::array<double, 3>;

D3 sub(const D3& a, const D3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
D3 cross3(const D3& a, const D3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
double dot3(const D3& a, const D3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// ---- the convex hull of a mesh (crates/dynamis-hull/src/hull.rs:53-288) ----
// Incremental quickhull in f32 with the reference's choices, so that its vertex numbering (which
// hull contacts carry as features and the warm start relays by) is the reference's: the initial
// tetrahedron from the x extremes, the point farthest from their line and the one farthest from
// that plane; each round expands the live face whose first outside point lies farthest (the last
// such face on ties), from its farthest outside point (again the last on ties); a face sees a point
// beyond 1e-6; the output keeps the surviving faces in creation order and numbers the vertices by
// first appearance over them. Faces live in one growing array; their outside sets are index lists.
struct HullBuild {
    const std::vector<std::array<float, 3>>& p;
    std::vector<std::array<uint32_t, 3>> corner;  // a, b, c of every face ever made
    std::vector<std::array<float, 4>> plane;      // unit normal, offset
    std::vector<std::vector<uint32_t>> outside;
    std::vector<uint8_t> live;
    std::vector<uint8_t> cornered;  // per point: a corner of some face made so far

    static float dotf(const std::array<float, 3>& a, const std::array<float, 3>& b) {
        return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    }
    std::array<float, 3> unit_normal(uint32_t a, uint32_t b, uint32_t c) const {
        const std::array<float, 3> u = {p[b][0] - p[a][0], p[b][1] - p[a][1], p[b][2] - p[a][2]};
        const std::array<float, 3> v = {p[c][0] - p[a][0], p[c][1] - p[a][1], p[c][2] - p[a][2]};
        const std::array<float, 3> n = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
        const float len = std::sqrt(dotf(n, n));
        if (len < 1e-12f) return {0.0f, 0.0f, 0.0f};
        return {n[0] / len, n[1] / len, n[2] / len};
    }
    uint32_t add_face(uint32_t a, uint32_t b, uint32_t c) {
        cornered[a] = cornered[b] = cornered[c] = 1;
        const std::array<float, 3> n = unit_normal(a, b, c);
        corner.push_back({a, b, c});
        plane.push_back({n[0], n[1], n[2], dotf(n, p[a])});
        outside.emplace_back();
        live.push_back(1);
        return (uint32_t)corner.size() - 1;
    }
    float height(uint32_t f, uint32_t point) const {
        const std::array<float, 3> n = {plane[f][0], plane[f][1], plane[f][2]};
        return dotf(n, p[point]) - plane[f][3];
    }
    // each point joins the outside set of the first live face that sees it. A point that is already
    // a corner of the hull joins none: in exact arithmetic no face sees it, and where rounding says
    // otherwise (a skinny face through near-duplicate points) the reference's rounds would pick it
    // again and again without end
    void assign(const std::vector<uint32_t>& points) {
        for (uint32_t q : points)
            for (uint32_t f = 0; f < (uint32_t)corner.size() && !cornered[q]; ++f)
                if (live[f] && height(f, q) > 1e-6f) {
                    outside[f].push_back(q);
                    break;
                }
    }
};

bool convex_hull_f32(const std::vector<std::array<float, 3>>& p, std::vector<uint32_t>* order,
                     std::vector<std::array<uint32_t, 3>>* faces_out) {
    const uint32_t n = (uint32_t)p.size();
    if (n < 4) return false;
    uint32_t lo = 0, hi = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (p[i][0] < p[lo][0]) lo = i;
        if (p[i][0] > p[hi][0]) hi = i;
    }
    if (lo == hi) {
        lo = 0;
        hi = n - 1;
    }
    const std::array<float, 3> axis = {p[hi][0] - p[lo][0], p[hi][1] - p[lo][1], p[hi][2] - p[lo][2]};
    const float axis_sq = HullBuild::dotf(axis, axis);
    uint32_t third = 0;
    float far = -1.0f;
    for (uint32_t i = 0; i < n; ++i) {
        const std::array<float, 3> d = {p[i][0] - p[lo][0], p[i][1] - p[lo][1], p[i][2] - p[lo][2]};
        const float t = axis_sq > 0.0f ? HullBuild::dotf(d, axis) / axis_sq : 0.0f;
        const std::array<float, 3> foot = {p[lo][0] + axis[0] * t, p[lo][1] + axis[1] * t, p[lo][2] + axis[2] * t};
        const std::array<float, 3> off = {p[i][0] - foot[0], p[i][1] - foot[1], p[i][2] - foot[2]};
        const float dist = std::sqrt(HullBuild::dotf(off, off));
        if (dist > far) {
            far = dist;
            third = i;
        }
    }
    if (!(far > 1e-6f)) return false;
    HullBuild h{p, {}, {}, {}, {}, std::vector<uint8_t>(n, 0)};
    const std::array<float, 3> base = h.unit_normal(lo, hi, third);
    const float base_offset = HullBuild::dotf(base, p[lo]);
    uint32_t fourth = 0;
    far = 0.0f;
    for (uint32_t i = 0; i < n; ++i) {
        const float dist = std::fabs(HullBuild::dotf(base, p[i]) - base_offset);
        if (dist > far) {
            far = dist;
            fourth = i;
        }
    }
    if (!(far > 1e-6f)) return false;
    std::array<float, 3> middle;
    for (int a = 0; a < 3; ++a) middle[a] = (p[lo][a] + p[hi][a] + p[third][a] + p[fourth][a]) * 0.25f;
    const uint32_t tet[4][3] = {{lo, hi, third}, {lo, hi, fourth}, {lo, third, fourth}, {hi, third, fourth}};
    for (const auto& t : tet) {
        const uint32_t f = h.add_face(t[0], t[1], t[2]);
        if (HullBuild::dotf({h.plane[f][0], h.plane[f][1], h.plane[f][2]}, middle) - h.plane[f][3] > 0.0f) {
            h.plane[f] = {-h.plane[f][0], -h.plane[f][1], -h.plane[f][2], -h.plane[f][3]};
            std::swap(h.corner[f][1], h.corner[f][2]);
        }
    }
    std::vector<uint32_t> everyone(n);
    for (uint32_t i = 0; i < n; ++i) everyone[i] = i;
    h.assign(everyone);
    for (;;) {
        int64_t seed = -1;
        float seed_height = 0.0f;
        for (uint32_t f = 0; f < (uint32_t)h.corner.size(); ++f) {
            if (!h.live[f] || h.outside[f].empty()) continue;
            const float lead = h.height(f, h.outside[f].front());
            if (seed < 0 || !(lead < seed_height)) {
                seed = f;
                seed_height = lead;
            }
        }
        if (seed < 0) break;
        const uint32_t s = (uint32_t)seed;
        uint32_t apex = h.outside[s][0];
        float apex_height = h.height(s, apex);
        for (size_t k = 1; k < h.outside[s].size(); ++k) {
            const float ht = h.height(s, h.outside[s][k]);
            if (!(ht < apex_height)) {
                apex = h.outside[s][k];
                apex_height = ht;
            }
        }
        std::vector<uint32_t> seen;
        for (uint32_t f = 0; f < (uint32_t)h.corner.size(); ++f)
            if (h.live[f] && f != s && h.height(f, apex) > 1e-6f) seen.push_back(f);
        seen.push_back(s);
        auto key = [](uint32_t a, uint32_t b) { return ((uint64_t)a << 32) | b; };
        std::vector<uint64_t> rims;
        for (uint32_t f : seen)
            for (int e = 0; e < 3; ++e) rims.push_back(key(h.corner[f][e], h.corner[f][(e + 1) % 3]));
        std::sort(rims.begin(), rims.end());
        std::vector<std::array<uint32_t, 2>> horizon;
        for (uint32_t f : seen)
            for (int e = 0; e < 3; ++e) {
                const uint32_t a = h.corner[f][e], b = h.corner[f][(e + 1) % 3];
                if (!std::binary_search(rims.begin(), rims.end(), key(b, a))) horizon.push_back({a, b});
            }
        if (horizon.empty()) return false;
        std::vector<uint32_t> orphans;
        for (uint32_t f : seen) {
            orphans.insert(orphans.end(), h.outside[f].begin(), h.outside[f].end());
            h.outside[f].clear();
            h.live[f] = 0;
        }
        orphans.push_back(apex);
        for (const auto& e : horizon) h.add_face(e[0], e[1], apex);
        h.assign(orphans);
    }
    std::vector<uint32_t> number(n, UINT32_MAX);
    order->clear();
    faces_out->clear();
    for (uint32_t f = 0; f < (uint32_t)h.corner.size(); ++f) {
        if (!h.live[f]) continue;
        for (uint32_t v : h.corner[f])
            if (number[v] == UINT32_MAX) {
                number[v] = (uint32_t)order->size();
                order->push_back(v);
            }
        faces_out->push_back({number[h.corner[f][0]], number[h.corner[f][1]], number[h.corner[f][2]]});
    }
    return faces_out->size() >= 4;
}

// crates/dynamis-hull/src/solid.rs:3-105 (f64 accumulation about the vertex mean)
void hull_solid(HullSource* h) {
    size_t nv = h->vertices.size() / 3;
    D3 apex = {0, 0, 0};
    for (size_t i = 0; i < nv; ++i)
        for (int a = 0; a < 3; ++a) apex[a] += (double)h->vertices[3 * i + a];
    for (int a = 0; a < 3; ++a) apex[a] /= (double)nv;
    auto shifted = [&](uint32_t v) {
        return D3{(double)h->vertices[3 * v] - apex[0], (double)h->vertices[3 * v + 1] - apex[1],
                  (double)h->vertices[3 * v + 2] - apex[2]};
    };
    auto squared = [](double a, double b, double c) { return (a * a + b * b + c * c + a * b + a * c + b * c) / 10.0; };
    auto mixed = [](double ax, double bx, double cx, double ay, double by, double cy) {
        return (2.0 * (ax * ay + bx * by + cx * cy) + ax * by + ay * bx + ax * cy + ay * cx + bx * cy + by * cx) / 20.0;
    };
    double volume = 0.0;
    double first[3] = {0, 0, 0};
    double second[6] = {0, 0, 0, 0, 0, 0};
    for (size_t t = 0; t + 2 < h->triangles.size(); t += 3) {
        D3 a = shifted(h->triangles[t]), b = shifted(h->triangles[t + 1]), c = shifted(h->triangles[t + 2]);
        if (dot3(cross3(a, b), c) < 0.0) std::swap(b, c);
        double s = dot3(a, cross3(b, c)) / 6.0;
        volume += s;
        for (int k = 0; k < 3; ++k) first[k] += s * (a[k] + b[k] + c[k]) / 4.0;
        second[0] += s * squared(a[0], b[0], c[0]);
        second[3] += s * squared(a[1], b[1], c[1]);
        second[5] += s * squared(a[2], b[2], c[2]);
        second[1] += s * mixed(a[0], b[0], c[0], a[1], b[1], c[1]);
        second[2] += s * mixed(a[0], b[0], c[0], a[2], b[2], c[2]);
        second[4] += s * mixed(a[1], b[1], c[1], a[2], b[2], c[2]);
    }
    double cen[3] = {first[0] / volume, first[1] / volume, first[2] / volume};
    h->volume = (float)volume;
    for (int k = 0; k < 3; ++k) h->centroid[k] = (float)(apex[k] + cen[k]);
    h->unit_second_moment[0] = (float)((second[0] - volume * cen[0] * cen[0]) / volume);
    h->unit_second_moment[1] = (float)((second[1] - volume * cen[0] * cen[1]) / volume);
    h->unit_second_moment[2] = (float)((second[2] - volume * cen[0] * cen[2]) / volume);
    h->unit_second_moment[3] = (float)((second[3] - volume * cen[1] * cen[1]) / volume);
    h->unit_second_moment[4] = (float)((second[4] - volume * cen[1] * cen[2]) / volume);
    h->unit_second_moment[5] = (float)((second[5] - volume * cen[2] * cen[2]) / volume);
}

// ---- mass properties (crates/dynamis-model/src/mass.rs) ----
struct Solid {
    float volume;
    float centroid[3];
    float second[6];
};
constexpr float kPi = 3.14159265358979323846f;

// analytic_solid / shape_solid (mass.rs:33-112) of a collider description's own, unscaled shape
bool analytic_solid(const dyn_collider_desc& c, const std::vector<HullSource>& hulls, Solid* s) {
    std::memset(s, 0, sizeof(*s));
    switch (c.shape) {
        case DYN_SHAPE_SPHERE: {
            float r = c.radius;
            float m = r * r / 5.0f;
            s->volume = 4.0f / 3.0f * kPi * r * r * r;
            s->second[0] = m;
            s->second[3] = m;
            s->second[5] = m;
            return true;
        }
        case DYN_SHAPE_CUBOID: {
            float ex = c.half_extents[0] * 2.0f, ey = c.half_extents[1] * 2.0f, ez = c.half_extents[2] * 2.0f;
            s->volume = ex * ey * ez;
            s->second[0] = ex * ex / 12.0f;
            s->second[3] = ey * ey / 12.0f;
            s->second[5] = ez * ez / 12.0f;
            return true;
        }
        case DYN_SHAPE_CAPSULE: {
            float r = c.radius, hh = c.half_height;
            float cyl = kPi * r * r * 2.0f * hh;
            float sph = 4.0f / 3.0f * kPi * r * r * r;
            float total = cyl + sph;
            float lateral = (cyl * r * r / 4.0f + sph * r * r / 5.0f) / total;
            float axial = (cyl * 4.0f * hh * hh / 12.0f + sph * (r * r / 5.0f + 3.0f / 4.0f * r * hh + hh * hh)) / total;
            s->volume = total;
            s->second[0] = lateral;
            s->second[3] = axial;
            s->second[5] = lateral;
            return true;
        }
        case DYN_SHAPE_CYLINDER: {
            float r = c.radius, height = c.half_height * 2.0f;
            float lateral = r * r / 4.0f;
            s->volume = kPi * r * r * height;
            s->second[0] = lateral;
            s->second[3] = height * height / 12.0f;
            s->second[5] = lateral;
            return true;
        }
        case DYN_SHAPE_HULL: {
            if (c.source >= hulls.size()) return false;
            const HullSource& h = hulls[c.source];
            s->volume = h.volume;
            for (int k = 0; k < 3; ++k) s->centroid[k] = h.centroid[k];
            for (int k = 0; k < 6; ++k) s->second[k] = h.unit_second_moment[k];
            return true;
        }
        default:
            return false;
    }
}

// crates/dynamis-model/src/math.rs:50-65 quat_rotate: v + 2 (s (u x v) + (u . v) u - (u . u) v)
void model_rotate(const float q[4], const float v[3], float out[3]) {
    const float ux = q[0], uy = q[1], uz = q[2], s = q[3];
    const float uv = ux * v[0] + uy * v[1] + uz * v[2];
    const float uu = ux * ux + uy * uy + uz * uz;
    const float cx = uy * v[2] - uz * v[1], cy = uz * v[0] - ux * v[2], cz = ux * v[1] - uy * v[0];
    out[0] = v[0] + 2.0f * (s * cx + uv * ux - uu * v[0]);
    out[1] = v[1] + 2.0f * (s * cy + uv * uy - uu * v[1]);
    out[2] = v[2] + 2.0f * (s * cz + uv * uz - uu * v[2]);
}

using M3 = std::array<std::array<float, 3>, 3>;
M3 mat_from_quat(const float q[4]) {
    float x = q[0], y = q[1], z = q[2], w = q[3];
    return M3{{{1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y - w * z), 2.0f * (x * z + w * y)},
               {2.0f * (x * y + w * z), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z - w * x)},
               {2.0f * (x * z - w * y), 2.0f * (y * z + w * x), 1.0f - 2.0f * (x * x + y * y)}}};
}
M3 mat_mul(const M3& a, const M3& b) {
    M3 r{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
    return r;
}

bool inertia_inverse(const float in[6], float out[6]) {
    float xx = in[0], xy = in[1], xz = in[2], yy = in[3], yz = in[4], zz = in[5];
    float cxx = yy * zz - yz * yz, cxy = xz * yz - xy * zz, cxz = xy * yz - xz * yy;
    float cyy = xx * zz - xz * xz, cyz = xy * xz - xx * yz, czz = xx * yy - xy * xy;
    float det = xx * cxx + xy * cxy + xz * cxz;
    if (!(xx > 0.0f && czz > 0.0f && det > 0.0f)) return false;
    out[0] = cxx / det;
    out[1] = cxy / det;
    out[2] = cxz / det;
    out[3] = cyy / det;
    out[4] = cyz / det;
    out[5] = czz / det;
    return true;
}

}  // namespace

void rebuild_rows(dyn_world* w) {
    if (w->raw_rows || !w->rows_dirty) return;
    const uint32_t ids = (uint32_t)w->spawn_states.size();
    w->removed.resize(ids, 0u);
    std::vector<uint32_t> order;
    order.reserve(ids);
    for (uint32_t i = 0; i < ids; ++i) {
        const dyn_body_descriptor_record& d = w->spawn_descs[i];
        if (!w->removed[i] && (d.flags & DYN_BODY_KINEMATIC) == 0u && d.inverse_mass > 0.0f) order.push_back(i);
    }
    w->dynamic_count = (uint32_t)order.size();
    for (uint32_t i = 0; i < ids; ++i) {
        const dyn_body_descriptor_record& d = w->spawn_descs[i];
        if (!w->removed[i] && !((d.flags & DYN_BODY_KINEMATIC) == 0u && d.inverse_mass > 0.0f)) order.push_back(i);
    }
    const uint32_t n = (uint32_t)order.size();
    w->states.resize(n);
    w->descs.resize(n);
    w->row_of_id.assign(ids, DYN_NO_BODY);
    for (uint32_t r = 0; r < n; ++r) {
        w->states[r] = w->spawn_states[order[r]];
        w->descs[r] = w->spawn_descs[order[r]];
        w->row_of_id[order[r]] = r;
    }
    w->body_world.assign(n, 0u);
    for (uint32_t r = 0; r < n; ++r) {
        if (order[r] < w->world_of_id.size()) w->body_world[r] = w->world_of_id[order[r]];
    }
    w->colliders.clear();
    w->owners.clear();
    for (size_t i = 0; i < w->spawn_owner.size(); ++i) {
        if (w->removed[w->spawn_owner[i]]) continue;
        w->colliders.push_back(w->spawn_colliders[i]);
        w->owners.push_back(w->row_of_id[w->spawn_owner[i]]);
    }
    w->rows_dirty = false;
    w->scene_dirty = true;  // whoever rebuilt the rows (an export, a read), the device needs them
}

std::vector<dyn_shape_source_record> shape_sources(const dyn_world* w, std::vector<float>* verts) {
    std::vector<dyn_shape_source_record> out(w->hulls.size());
    verts->clear();
    for (size_t s = 0; s < w->hulls.size(); ++s) {
        const HullSource& h = w->hulls[s];
        dyn_shape_source_record& r = out[s];
        std::memset(&r, 0, sizeof(r));
        r.kind = DYN_SHAPE_HULL;
        r.vertex_offset = (uint32_t)(verts->size() / 4);
        r.vertex_count = (uint32_t)(h.vertices.size() / 3);
        float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (size_t i = 0; i + 2 < h.vertices.size(); i += 3) {
            for (int a = 0; a < 3; ++a) {
                mn[a] = std::min(mn[a], h.vertices[i + a]);
                mx[a] = std::max(mx[a], h.vertices[i + a]);
                verts->push_back(h.vertices[i + a]);
            }
            verts->push_back(0.0f);
        }
        for (int a = 0; a < 3; ++a) {
            r.local_min[a] = mn[a];
            r.local_max[a] = mx[a];
        }
    }
    return out;
}


// ---- joint solve order (crates/dynamis-world/src/schedule.rs:105-296) ----
namespace {
uint32_t plan_find(std::vector<uint32_t>& roots, uint32_t row) {
    while (roots[row] != row) {
        roots[row] = roots[roots[row]];
        row = roots[row];
    }
    return row;
}
}  // namespace

void plan_joints(const std::vector<uint32_t>& first, const std::vector<uint32_t>& second, uint32_t body_rows,
                 uint32_t dynamic_count, JointPlan* plan) {
    constexpr uint32_t kNone = 0xFFFFFFFFu;
    const uint32_t joints = (uint32_t)first.size();
    plan->rows.clear();
    plan->layers.clear();
    plan->components.clear();
    plan->groups.clear();
    if (joints == 0) return;
    // components by union of the two ends; a row that does not simulate anchors its component
    std::vector<uint8_t> anchor(body_rows, 0);
    std::vector<uint32_t> roots(body_rows);
    for (uint32_t i = 0; i < body_rows; ++i) roots[i] = i;
    for (uint32_t j = 0; j < joints; ++j) {
        uint32_t a = first[j], b = second[j];
        if (a >= dynamic_count) anchor[a] = 1;
        if (b >= dynamic_count) anchor[b] = 1;
        uint32_t ra = plan_find(roots, a), rb = plan_find(roots, b);
        uint32_t root = std::min(ra, rb);
        roots[ra] = root;
        roots[rb] = root;
    }
    std::vector<uint32_t> root_of(joints);
    for (uint32_t j = 0; j < joints; ++j) root_of[j] = plan_find(roots, first[j]);
    std::vector<uint8_t> anchored(body_rows, 0);
    std::vector<uint32_t> head_of(body_rows, kNone);
    for (uint32_t j = 0; j < joints; ++j) {
        uint32_t r = root_of[j];
        anchored[r] |= (uint8_t)(anchor[first[j]] | anchor[second[j]]);
        head_of[r] = std::min(head_of[r], std::min(first[j], second[j]));
    }
    std::vector<std::vector<uint32_t>> adjacency(body_rows);
    for (uint32_t j = 0; j < joints; ++j) {
        adjacency[first[j]].push_back(second[j]);
        adjacency[second[j]].push_back(first[j]);
    }
    // depth: breadth-first from the anchors, then from the head of each unanchored component
    std::vector<uint32_t> depth(body_rows, kNone);
    std::vector<uint32_t> frontier;
    for (uint32_t b = 0; b < body_rows; ++b) {
        if (anchor[b]) {
            depth[b] = 0;
            frontier.push_back(b);
        }
    }
    for (uint32_t r = 0; r < body_rows; ++r) {
        if (head_of[r] != kNone && !anchored[r]) {
            depth[head_of[r]] = 0;
            frontier.push_back(head_of[r]);
        }
    }
    for (size_t cursor = 0; cursor < frontier.size(); ++cursor) {
        uint32_t b = frontier[cursor];
        for (uint32_t nb : adjacency[b]) {
            if (depth[nb] == kNone) {
                depth[nb] = depth[b] + 1;
                frontier.push_back(nb);
            }
        }
    }
    // joints in order of depth, component, row; each takes the layer after its ends' last layers
    std::vector<uint32_t> settled(joints);
    for (uint32_t j = 0; j < joints; ++j) settled[j] = j;
    auto depth_key = [&](uint32_t j) { return std::max(depth[first[j]], depth[second[j]]); };
    std::sort(settled.begin(), settled.end(), [&](uint32_t x, uint32_t y) {
        uint32_t dx = depth_key(x), dy = depth_key(y);
        if (dx != dy) return dx < dy;
        if (root_of[x] != root_of[y]) return root_of[x] < root_of[y];
        return x < y;
    });
    std::vector<uint32_t> held_layer(body_rows, 0);
    struct Held {
        uint32_t root, layer, row;
    };
    std::vector<Held> held;
    held.reserve(joints);
    for (uint32_t j : settled) {
        uint32_t layer = std::max(held_layer[first[j]], held_layer[second[j]]) + 1;
        held_layer[first[j]] = layer;
        held_layer[second[j]] = layer;
        held.push_back(Held{root_of[j], layer, j});
    }
    std::sort(held.begin(), held.end(), [](const Held& x, const Held& y) {
        if (x.root != y.root) return x.root < y.root;
        if (x.layer != y.layer) return x.layer < y.layer;
        return x.row < y.row;
    });
    struct Comp {
        uint32_t first_layer, layers, first_row, head, lanes;
    };
    std::vector<uint32_t> rows, layers;
    std::vector<Comp> comps;
    size_t index = 0;
    while (index < held.size()) {
        uint32_t root = held[index].root;
        Comp c{(uint32_t)(layers.size() / 2), 0, (uint32_t)rows.size(), kNone, 0};
        uint32_t widest = 0;
        while (index < held.size() && held[index].root == root) {
            uint32_t layer = held[index].layer;
            size_t start = rows.size();
            while (index < held.size() && held[index].root == root && held[index].layer == layer) {
                uint32_t j = held[index].row;
                c.head = std::min(c.head, std::min(first[j], second[j]));
                rows.push_back(j);
                ++index;
            }
            uint32_t count = (uint32_t)(rows.size() - start);
            widest = std::max(widest, count);
            layers.push_back((uint32_t)start);
            layers.push_back(count);
            c.layers += 1;
        }
        uint32_t lanes = 1;
        while (lanes < widest) lanes <<= 1;
        c.lanes = std::min(lanes, 64u);  // JOINT_BATCH_LANES
        comps.push_back(c);
    }
    std::stable_sort(comps.begin(), comps.end(), [](const Comp& x, const Comp& y) {
        if (x.lanes != y.lanes) return x.lanes > y.lanes;
        if (x.layers != y.layers) return x.layers > y.layers;
        return x.head < y.head;
    });
    for (const Comp& c : comps) {
        plan->components.push_back((uint32_t)(plan->layers.size() / 2));
        plan->components.push_back(c.layers);
        uint32_t cursor = c.first_row;
        for (uint32_t l = c.first_layer; l < c.first_layer + c.layers; ++l) {
            uint32_t count = layers[2 * l + 1];
            plan->layers.push_back((uint32_t)plan->rows.size());
            plan->layers.push_back(count);
            plan->rows.insert(plan->rows.end(), rows.begin() + cursor, rows.begin() + cursor + count);
            cursor += count;
        }
    }
    // device packing (not the reference's workgroup packing: results do not depend on it, since
    // components share no body): consecutive components of equal lane width share a 32-lane warp,
    // at most kComponentsPerWarp of them. A component is a chain of dependent solves, so a pass
    // takes (layers x latency of one solve); spreading components over more warps gives each SM
    // several warps to interleave instead of one warp holding 32 chains.
    constexpr uint32_t kComponentsPerWarp = 8;
    uint32_t c = 0;
    while (c < (uint32_t)comps.size()) {
        uint32_t lanes = std::min(comps[c].lanes, 32u);
        uint32_t span = comps[c].layers;
        uint32_t taken = 1;
        while (c + taken < (uint32_t)comps.size() && taken < kComponentsPerWarp && (taken + 1) * lanes <= 32u &&
               std::min(comps[c + taken].lanes, 32u) == lanes) {
            span = std::max(span, comps[c + taken].layers);
            ++taken;
        }
        plan->groups.push_back(c);
        plan->groups.push_back(taken);
        plan->groups.push_back(lanes);
        plan->groups.push_back(span);
        c += taken;
    }
}

dyn_status rebuild_joints(dyn_world* w) {
    rebuild_rows(w);
    const uint32_t m = (uint32_t)w->joint_descs.size();
    const uint32_t n = (uint32_t)w->states.size();
    w->joint_rows.resize(m);
    std::vector<uint32_t> first(m), second(m);
    for (uint32_t j = 0; j < m; ++j) {
        const dyn_constraint_descriptor_record& d = w->joint_descs[j];
        uint32_t a = d.first_body_id < w->row_of_id.size() ? w->row_of_id[d.first_body_id] : DYN_NO_BODY;
        uint32_t b = d.second_body_id < w->row_of_id.size() ? w->row_of_id[d.second_body_id] : DYN_NO_BODY;
        if (a == DYN_NO_BODY || b == DYN_NO_BODY || a >= n || b >= n)
            return fail(w, DYN_ERR_INVALID, "a joint must join two live bodies");
        if (a < w->body_world.size() && b < w->body_world.size() && w->body_world[a] != w->body_world[b])
            return fail(w, DYN_ERR_INVALID, "a joint must not join bodies of different sub-worlds");
        w->joint_rows[j] = dyn_constraint_rows_record{a, b};
        first[j] = a;
        second[j] = b;
    }
    plan_joints(first, second, n, w->dynamic_count, &w->joint_plan);
    return DYN_OK;
}
}  // namespace dyn

using namespace dyn;

extern "C" {

DYN_API uint32_t dyn_abi_version(void) { return 1u; }

DYN_API const char* dyn_status_string(dyn_status s) {
    switch (s) {
        case DYN_OK: return "ok";
        case DYN_ERR_INVALID: return "invalid argument";
        case DYN_ERR_CAPACITY: return "capacity exceeded";
        case DYN_ERR_CUDA: return "CUDA runtime error";
        case DYN_ERR_NO_DEVICE: return "no CUDA device";
        case DYN_ERR_DEVICE_STATUS: return "device gave up a bounded wait";
        case DYN_ERR_DEGENERATE: return "degenerate hull";
        case DYN_NOT_READY: return "no observation completed yet";
        default: return "unknown status";
    }
}

DYN_API void dyn_config_default(dyn_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->gravity[1] = -9.81f;
    c->damping = 0.05f;
    c->angular_damping = 0.05f;
    c->substeps = 2;
    c->solve_iterations = 8;
    c->position_iterations = 10;
    c->relaxation = 0.8f;
    c->slop = 0.005f;
    c->contact_margin = 0.02f;
    c->restitution_threshold = 1.0f;
    c->max_velocity = 200.0f;
    c->max_angular_velocity = 400.0f;
    c->sleep_velocity = 0.2f;
    c->sleep_angular_velocity = 0.5f;
    c->sleep_time = 0.5f;
    c->friction_combine = 0;     // Multiply
    c->restitution_combine = 2;  // Max
}

DYN_API void dyn_collider_desc_default(dyn_collider_desc* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->shape = DYN_SHAPE_SPHERE;
    c->radius = 0.5f;
    c->rotation[3] = 1.0f;
    c->scale[0] = c->scale[1] = c->scale[2] = 1.0f;
    c->friction = 0.5f;
    c->contact_frequency = INFINITY;
    c->contact_damping_ratio = 1.0f;
    c->collision_group = DYN_NO_COLLISION_FILTER;
    c->collision_mask = DYN_NO_COLLISION_FILTER;
    c->impact_force = INFINITY;
}

DYN_API void dyn_body_desc_default(dyn_body_desc* b) {
    if (!b) return;
    std::memset(b, 0, sizeof(*b));
    b->orientation[3] = 1.0f;
    b->mass = 1.0f;
    b->gravity_scale = 1.0f;
    b->linear_damping = -1.0f;
    b->angular_damping = -1.0f;
    b->sleep_velocity = -1.0f;
    b->sleep_angular_velocity = -1.0f;
    b->collision_group = 1u;
    b->collision_mask = 0xFFFFFFFFu;
}

DYN_API const char* dyn_last_error(const dyn_world* w) { return w ? w->last_error.c_str() : "null world"; }

namespace {
// A hull source from its vertices and outward triangles; checks that it encloses a volume.
dyn_status store_hull(dyn_world* w, const std::vector<std::array<float, 3>>& vertices,
                      const std::vector<std::array<uint32_t, 3>>& triangles, uint32_t* out_source) {
    HullSource h;
    for (const auto& v : vertices) h.vertices.insert(h.vertices.end(), v.begin(), v.end());
    for (const auto& t : triangles) h.triangles.insert(h.triangles.end(), t.begin(), t.end());
    hull_solid(&h);
    if (!(h.volume > 0.0f) || !std::isfinite(h.volume)) return fail(w, DYN_ERR_DEGENERATE, "a hull must enclose a positive volume");
    *out_source = (uint32_t)w->hulls.size();
    w->hulls.push_back(std::move(h));
    return DYN_OK;
}
// hull() of crates/dynamis-hull/src/hull.rs:53-86: the referenced vertices in ascending index
// order, hulled, renumbered by first appearance over the surviving faces
dyn_status hull_from_points(dyn_world* w, const float* xyz, const std::vector<uint32_t>& used, uint32_t* out_source) {
    std::vector<std::array<float, 3>> pts;
    for (uint32_t i : used) {
        for (int a = 0; a < 3; ++a)
            if (!std::isfinite(xyz[3 * i + a])) return fail(w, DYN_ERR_INVALID, "a mesh vertex must be finite");
        pts.push_back({xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]});
    }
    std::vector<uint32_t> order;
    std::vector<std::array<uint32_t, 3>> faces;
    if (!convex_hull_f32(pts, &order, &faces)) return fail(w, DYN_ERR_DEGENERATE, "hull mesh points span no volume");
    std::vector<std::array<float, 3>> vertices;
    for (uint32_t v : order) vertices.push_back(pts[v]);
    return store_hull(w, vertices, faces, out_source);
}
}  // namespace

DYN_API dyn_status dyn_add_hull(dyn_world* w, const float* xyz, uint32_t n, uint32_t* out_source) {
    if (!w || !xyz || !out_source) return fail(w, DYN_ERR_INVALID, "dyn_add_hull: null argument");
    std::vector<uint32_t> all(n);
    for (uint32_t i = 0; i < n; ++i) all[i] = i;
    return hull_from_points(w, xyz, all, out_source);
}

DYN_API dyn_status dyn_add_hull_from_mesh(dyn_world* w, const float* xyz, uint32_t nv, const uint32_t* triangles, uint32_t nt,
                                          uint32_t* out_source) {
    if (!w || !xyz || !triangles || !out_source) return fail(w, DYN_ERR_INVALID, "dyn_add_hull_from_mesh: null argument");
    if (nt == 0) return fail(w, DYN_ERR_INVALID, "a mesh must carry at least one triangle");
    std::vector<uint8_t> referenced(nv, 0);
    for (uint64_t t = 0; t < 3ull * nt; ++t) {
        if (triangles[t] >= nv) return fail(w, DYN_ERR_INVALID, "a mesh triangle must reference the vertices of its own mesh");
        referenced[triangles[t]] = 1;
    }
    std::vector<uint32_t> used;
    for (uint32_t i = 0; i < nv; ++i)
        if (referenced[i]) used.push_back(i);
    return hull_from_points(w, xyz, used, out_source);
}

DYN_API dyn_status dyn_add_hull_mesh(dyn_world* w, const float* xyz, uint32_t nv, const uint32_t* triangles, uint32_t nt,
                                     uint32_t* out_source) {
    if (!w || !xyz || !triangles || !out_source) return fail(w, DYN_ERR_INVALID, "dyn_add_hull_mesh: null argument");
    if (nt == 0 || nv == 0) return fail(w, DYN_ERR_INVALID, "a hull must contain vertices and triangles");
    std::vector<std::array<float, 3>> vertices(nv);
    for (uint32_t i = 0; i < nv; ++i)
        for (int a = 0; a < 3; ++a) {
            if (!std::isfinite(xyz[3 * i + a])) return fail(w, DYN_ERR_INVALID, "a mesh vertex must be finite");
            vertices[i][a] = xyz[3 * i + a];
        }
    std::vector<std::array<uint32_t, 3>> tris(nt);
    for (uint32_t t = 0; t < nt; ++t)
        for (int a = 0; a < 3; ++a) {
            if (triangles[3 * t + a] >= nv) return fail(w, DYN_ERR_INVALID, "a mesh triangle must reference the vertices of its own mesh");
            tris[t][a] = triangles[3 * t + a];
        }
    return store_hull(w, vertices, tris, out_source);
}

DYN_API dyn_status dyn_hull_info(const dyn_world* w, uint32_t source, uint32_t* vc, uint32_t* tc, float* volume,
                                 float centroid[3]) {
    if (!w || source >= w->hulls.size()) return DYN_ERR_INVALID;
    const HullSource& h = w->hulls[source];
    if (vc) *vc = (uint32_t)(h.vertices.size() / 3);
    if (tc) *tc = (uint32_t)(h.triangles.size() / 3);
    if (volume) *volume = h.volume;
    if (centroid)
        for (int k = 0; k < 3; ++k) centroid[k] = h.centroid[k];
    return DYN_OK;
}

DYN_API dyn_status dyn_spawn_bodies(dyn_world* w, const dyn_body_desc* bodies, uint32_t n, const dyn_collider_desc* cols,
                                    uint32_t k, uint32_t* out_ids) {
    if (!w || (n && !bodies)) return fail(w, DYN_ERR_INVALID, "dyn_spawn_bodies: null argument");
    if (w->raw_rows) return fail(w, DYN_ERR_INVALID, "dyn_spawn_bodies: scene was replaced by dyn_upload_bodies");
    for (uint32_t b = 0; b < n; ++b) {
        const dyn_body_desc& bd = bodies[b];
        if (bd.collider_count == 0 || (uint64_t)bd.collider_first + bd.collider_count > k || !cols)
            return fail(w, DYN_ERR_INVALID, "dyn_spawn_bodies: a body requires at least one collider in range");
        if (bd.kinematic && bd.ccd) return fail(w, DYN_ERR_INVALID, "dyn_spawn_bodies: kinematic bodies cannot declare ccd");
        uint32_t body_id = (uint32_t)w->spawn_states.size();
        // ColliderRecord::build for each collider
        std::vector<dyn_collider_record> recs;
        for (uint32_t c = 0; c < bd.collider_count; ++c) {
            const dyn_collider_desc& cd = cols[bd.collider_first + c];
            dyn_collider_record r;
            std::memset(&r, 0, sizeof(r));
            r.slot = (uint32_t)(w->spawn_colliders.size() + recs.size());
            r.kind = cd.shape;
            if (cd.shape == DYN_SHAPE_HULL && cd.source >= w->hulls.size())
                return fail(w, DYN_ERR_INVALID, "dyn_spawn_bodies: unknown hull source");
            if (cd.shape == DYN_SHAPE_NONE || cd.shape > DYN_SHAPE_PLANE || cd.shape == DYN_SHAPE_MESH
                || cd.shape == DYN_SHAPE_HEIGHTFIELD || cd.shape == DYN_SHAPE_TRIANGLE)
                return fail(w, DYN_ERR_INVALID, "dyn_spawn_bodies: shape outside the step path");
            uint32_t flags = cd.sensor ? DYN_COLLIDER_SENSOR : 0u;
            flags |= cd.events & (DYN_EVENT_MODE_BEGIN_END | DYN_EVENT_MODE_PERSIST);
            if (cd.events & DYN_EVENT_MODE_PERSIST) flags |= DYN_EVENT_MODE_BEGIN_END;
            r.flags = flags;
            // ShapeScale (crates/dynamis-abi/src/shape.rs:48-193): round shapes fold a uniform scale
            // into their dimensions and keep any other in the record; cuboids scale their extents;
            // hulls keep theirs in the record; planes take none
            const bool round = cd.shape == DYN_SHAPE_SPHERE || cd.shape == DYN_SHAPE_CAPSULE || cd.shape == DYN_SHAPE_CYLINDER;
            const bool uniform = cd.scale[0] == cd.scale[1] && cd.scale[1] == cd.scale[2];
            const float fold = round && uniform ? cd.scale[0] : 1.0f;
            r.radius = round ? cd.radius * fold : 0.0f;
            r.half_height = (cd.shape == DYN_SHAPE_CAPSULE || cd.shape == DYN_SHAPE_CYLINDER) ? cd.half_height * fold : 0.0f;
            r.impact_force = cd.impact_force;
            if (cd.shape == DYN_SHAPE_CUBOID) {
                for (int a = 0; a < 3; ++a) r.half_extents[a] = cd.half_extents[a] * cd.scale[a];
            }
            r.collision_group = cd.collision_group;
            r.collision_mask = cd.collision_mask;
            for (int a = 0; a < 3; ++a) r.local_offset[a] = cd.offset[a];
            for (int a = 0; a < 4; ++a) r.local_rotation[a] = cd.rotation[a];
            r.friction = cd.friction;
            r.restitution = cd.restitution;
            r.source = cd.shape == DYN_SHAPE_HULL ? cd.source : 0u;
            r.rolling_friction = cd.rolling_friction;
            const bool in_record = cd.shape == DYN_SHAPE_HULL || (round && !uniform);
            for (int a = 0; a < 3; ++a) r.scale[a] = in_record ? cd.scale[a] : 1.0f;
            r.spin_friction = cd.spin_friction;
            r.relaxation = std::isinf(cd.contact_frequency) ? 0.0f : 1.0f / (6.28318530717958647692f * cd.contact_frequency);
            r.damping_ratio = cd.contact_damping_ratio;
            recs.push_back(r);
        }
        // mass properties (mass.rs:155-212) over non-sensor solids
        struct Item {
            const dyn_collider_record* c;
            const dyn_collider_desc* d;
            Solid s;
            float volume;
        };
        std::vector<Item> items;
        for (uint32_t c = 0; c < bd.collider_count; ++c) {
            const dyn_collider_desc& cd = cols[bd.collider_first + c];
            if (cd.sensor) continue;
            Solid s;
            if (!analytic_solid(cd, w->hulls, &s)) continue;
            items.push_back(Item{&recs[c], &cd, s, cd.scale[0] * cd.scale[1] * cd.scale[2] * s.volume});
        }
        float total_volume = 0.0f;
        for (const Item& it : items) total_volume += it.volume;
        bool density_mode = bd.density > 0.0f;
        float mass = density_mode ? bd.density * total_volume : bd.mass;
        bool dynamic = !bd.kinematic && mass > 0.0f;
        float com[3] = {0, 0, 0}, inertia[6] = {0, 0, 0, 0, 0, 0}, inv_inertia[6] = {0, 0, 0, 0, 0, 0};
        if (!items.empty() && total_volume > 0.0f && mass > 0.0f) {
            auto centroid_of = [&](const Item& it, float out[3]) {
                float sc[3];
                for (int a = 0; a < 3; ++a) sc[a] = it.d->scale[a] * it.s.centroid[a];
                float rot[3];
                model_rotate(it.d->rotation, sc, rot);
                for (int a = 0; a < 3; ++a) out[a] = it.d->offset[a] + rot[a];
            };
            float sum[3] = {0, 0, 0};
            for (const Item& it : items) {
                float at[3];
                centroid_of(it, at);
                for (int a = 0; a < 3; ++a) sum[a] += at[a] * it.volume;
            }
            for (int a = 0; a < 3; ++a) com[a] = sum[a] / total_volume;
            float second[6] = {0, 0, 0, 0, 0, 0};
            for (const Item& it : items) {
                float shape_mass = mass * it.volume / total_volume;
                const float* u = it.s.second;
                const float* sc = it.d->scale;
                float local[6] = {u[0] * sc[0] * sc[0], u[1] * sc[0] * sc[1], u[2] * sc[0] * sc[2],
                                  u[3] * sc[1] * sc[1], u[4] * sc[1] * sc[2], u[5] * sc[2] * sc[2]};
                M3 r = mat_from_quat(it.d->rotation);
                M3 s = {{{local[0], local[1], local[2]}, {local[1], local[3], local[4]}, {local[2], local[4], local[5]}}};
                M3 rt = {{{r[0][0], r[1][0], r[2][0]}, {r[0][1], r[1][1], r[2][1]}, {r[0][2], r[1][2], r[2][2]}}};
                M3 m = mat_mul(r, mat_mul(s, rt));
                float rotated[6] = {m[0][0], (m[0][1] + m[1][0]) * 0.5f, (m[0][2] + m[2][0]) * 0.5f,
                                    m[1][1], (m[1][2] + m[2][1]) * 0.5f, m[2][2]};
                float at[3];
                centroid_of(it, at);
                float d[3] = {at[0] - com[0], at[1] - com[1], at[2] - com[2]};
                float tr[6] = {rotated[0] + d[0] * d[0], rotated[1] + d[0] * d[1], rotated[2] + d[0] * d[2],
                               rotated[3] + d[1] * d[1], rotated[4] + d[1] * d[2], rotated[5] + d[2] * d[2]};
                for (int q = 0; q < 6; ++q) second[q] += tr[q] * shape_mass;
            }
            float xx = second[0], xy = second[1], xz = second[2], yy = second[3], yz = second[4], zz = second[5];
            float I[6] = {yy + zz, -xy, -xz, xx + zz, -yz, xx + yy};
            for (int q = 0; q < 6; ++q) inertia[q] = I[q];
            if (!inertia_inverse(inertia, inv_inertia))
                return fail(w, DYN_ERR_INVALID, "dyn_spawn_bodies: inertia tensor must be positive definite");
        }
        dyn_body_descriptor_record d;
        std::memset(&d, 0, sizeof(d));
        d.inverse_mass = dynamic ? 1.0f / mass : 0.0f;
        d.linear_damping = bd.linear_damping >= 0.0f ? bd.linear_damping : w->config.damping;
        d.angular_damping = bd.angular_damping >= 0.0f ? bd.angular_damping : w->config.angular_damping;
        d.gravity_scale = bd.gravity_scale;
        d.sleep_velocity = bd.sleep_velocity >= 0.0f ? bd.sleep_velocity : 0.0f;
        d.sleep_angular_velocity = bd.sleep_angular_velocity >= 0.0f ? bd.sleep_angular_velocity : 0.0f;
        uint32_t flags = 0;
        if (bd.kinematic) flags |= DYN_BODY_KINEMATIC;
        if (bd.ccd) flags |= DYN_BODY_CCD;
        if (bd.sleep_velocity >= 0.0f) flags |= DYN_OVERRIDE_SLEEP_LINEAR;
        if (bd.sleep_angular_velocity >= 0.0f) flags |= DYN_OVERRIDE_SLEEP_ANGULAR;
        d.flags = flags;
        d.collision_group = bd.collision_group;
        d.collision_mask = bd.collision_mask;
        for (int a = 0; a < 3; ++a) d.com[a] = com[a];
        for (int q = 0; q < 6; ++q) {
            d.inertia[q] = inertia[q];
            d.inverse_inertia[q] = inv_inertia[q];
        }
        dyn_body_state_record s;
        std::memset(&s, 0, sizeof(s));
        for (int a = 0; a < 3; ++a) {
            s.position[a] = bd.position[a];
            s.prev_position[a] = bd.position[a];
            s.velocity[a] = bd.velocity[a];
            s.angular_velocity[a] = bd.angular_velocity[a];
        }
        for (int a = 0; a < 4; ++a) {
            s.orientation[a] = bd.orientation[a];
            s.prev_orientation[a] = bd.orientation[a];
        }
        s.body_id = body_id;
        s.generation = 0;
        w->spawn_states.push_back(s);
        w->spawn_descs.push_back(d);
        for (const dyn_collider_record& r : recs) {
            w->spawn_colliders.push_back(r);
            w->spawn_owner.push_back(body_id);
        }
        if (out_ids) out_ids[b] = body_id;
    }
    w->rows_dirty = true;
    return DYN_OK;
}

DYN_API dyn_status dyn_scene_sizes(const dyn_world* cw, uint32_t* bodies, uint32_t* dyn_bodies, uint32_t* colliders,
                                   uint32_t* sources, uint32_t* vertices) {
    if (!cw) return DYN_ERR_INVALID;
    dyn_world* w = const_cast<dyn_world*>(cw);
    rebuild_rows(w);
    if (bodies) *bodies = (uint32_t)w->states.size();
    if (dyn_bodies) *dyn_bodies = w->dynamic_count;
    if (colliders) *colliders = (uint32_t)w->colliders.size();
    if (sources) *sources = (uint32_t)w->hulls.size();
    if (vertices) {
        uint32_t v = 0;
        for (const HullSource& h : w->hulls) v += (uint32_t)(h.vertices.size() / 3);
        *vertices = v;
    }
    return DYN_OK;
}

DYN_API dyn_status dyn_export_scene(const dyn_world* cw, dyn_body_state_record* states, dyn_body_descriptor_record* descs,
                                    dyn_collider_record* colliders, uint32_t* owners, dyn_shape_source_record* sources,
                                    float* vertices) {
    if (!cw) return DYN_ERR_INVALID;
    dyn_world* w = const_cast<dyn_world*>(cw);
    rebuild_rows(w);
    if (states) std::memcpy(states, w->states.data(), w->states.size() * sizeof(*states));
    if (descs) std::memcpy(descs, w->descs.data(), w->descs.size() * sizeof(*descs));
    if (colliders) std::memcpy(colliders, w->colliders.data(), w->colliders.size() * sizeof(*colliders));
    if (owners) std::memcpy(owners, w->owners.data(), w->owners.size() * sizeof(*owners));
    std::vector<float> verts;
    std::vector<dyn_shape_source_record> src = shape_sources(w, &verts);
    if (sources) std::memcpy(sources, src.data(), src.size() * sizeof(*sources));
    if (vertices) std::memcpy(vertices, verts.data(), verts.size() * sizeof(float));
    return DYN_OK;
}

DYN_API dyn_status dyn_step_params_for(const dyn_world* cw, float dt, dyn_step_params* out) {
    if (!cw || !out) return DYN_ERR_INVALID;
    if (!(dt > 0.0f) || !std::isfinite(dt)) return fail(const_cast<dyn_world*>(cw), DYN_ERR_INVALID, "a step timestep must be positive");
    dyn_world* w = const_cast<dyn_world*>(cw);
    rebuild_rows(w);
    const dyn_config& c = w->config;
    std::memset(out, 0, sizeof(*out));
    out->gravity[0] = c.gravity[0];
    out->gravity[1] = c.gravity[1];
    out->gravity[2] = c.gravity[2];
    out->dt = dt;
    out->substep_dt = dt / (float)c.substeps;
    out->damping = c.damping;
    out->angular_damping = c.angular_damping;
    out->body_count = (uint32_t)w->states.size();
    out->substeps = c.substeps;
    out->solve_iterations = c.solve_iterations;
    out->relaxation = c.relaxation;
    out->slop = c.slop;
    out->restitution_threshold = c.restitution_threshold;
    out->max_velocity = c.max_velocity;
    out->max_angular_velocity = c.max_angular_velocity;
    out->dynamic_count = w->dynamic_count;
    out->sleep_velocity = c.sleep_velocity;
    out->sleep_angular_velocity = c.sleep_angular_velocity;
    out->sleep_time = c.sleep_time;
    out->friction_combine = c.friction_combine;
    out->restitution_combine = c.restitution_combine;
    out->position_iterations = c.position_iterations;
    out->contact_margin = c.contact_margin;
    out->collider_count = (uint32_t)w->colliders.size();
    out->constraint_count = (uint32_t)w->joint_descs.size();
    out->soft_iterations = 1;
    out->soft_substeps = 4;
    out->soft_substep_dt = dt / 4.0f;
    out->settle_velocity = 1.0e-4f;
    return DYN_OK;
}

// ---- constraints (ball joints) ----
namespace {
dyn_status add_constraint_record(dyn_world* w, const dyn_constraint_descriptor_record& r) {
    const uint32_t supported = DYN_CONSTRAINT_DISABLE_COLLISIONS | DYN_CONSTRAINT_WARM_START | DYN_CONSTRAINT_HAS_BREAK;
    if (r.kind != DYN_CONSTRAINT_BALL) return fail(w, DYN_ERR_INVALID, "only ball joints are on this path");
    if (r.flags & ~supported) return fail(w, DYN_ERR_INVALID, "ball joint limits and swing cones are not on this path");
    uint32_t ids = (uint32_t)std::max(w->spawn_states.size(), w->row_of_id.size());
    if (r.first_body_id >= ids || r.second_body_id >= ids) return fail(w, DYN_ERR_INVALID, "a joint must join two live bodies");
    if (r.first_body_id == r.second_body_id) return fail(w, DYN_ERR_INVALID, "a joint must join two different bodies");
    for (int i = 0; i < 3; ++i) {
        if (!std::isfinite(r.anchor_a[i]) || !std::isfinite(r.anchor_b[i])) return fail(w, DYN_ERR_INVALID, "joint anchors must be finite");
    }
    w->joint_descs.push_back(r);
    dyn_constraint_runtime_record rt;
    std::memset(&rt, 0, sizeof(rt));
    rt.constraint_id = (uint32_t)w->joint_descs.size() - 1u;  // ConstraintRuntimeRecord::fresh
    w->joint_runtime.push_back(rt);
    w->joints_dirty = true;
    return DYN_OK;
}
}  // namespace

DYN_API dyn_status dyn_add_ball_joint(dyn_world* w, uint32_t first_body, uint32_t second_body, const float* anchor_a,
                                      const float* anchor_b, uint32_t* out_id) {
    if (!w || !anchor_a || !anchor_b) return fail(w, DYN_ERR_INVALID, "dyn_add_ball_joint: null argument");
    // ConstraintDesc::ball with the defaults of ConstraintDesc::VACANT, packed as
    // ConstraintDescriptorRecord::build does (crates/dynamis-abi/src/constraint.rs:109-141)
    dyn_constraint_descriptor_record r;
    std::memset(&r, 0, sizeof(r));
    r.kind = DYN_CONSTRAINT_BALL;
    r.first_body_id = first_body;
    r.second_body_id = second_body;
    r.flags = DYN_CONSTRAINT_DISABLE_COLLISIONS | DYN_CONSTRAINT_WARM_START;
    for (int i = 0; i < 3; ++i) {
        r.anchor_a[i] = anchor_a[i];
        r.anchor_b[i] = anchor_b[i];
    }
    r.axis_a[1] = 1.0f;
    r.swing_a = 3.14159265358979323846f;
    r.swing_b = 3.14159265358979323846f;
    r.gear_ratio = 1.0f;
    dyn_status st = add_constraint_record(w, r);
    if (st) return st;
    if (out_id) *out_id = (uint32_t)w->joint_descs.size() - 1u;
    return DYN_OK;
}

DYN_API dyn_status dyn_add_constraints(dyn_world* w, const dyn_constraint_descriptor_record* records, uint32_t m,
                                       uint32_t* out_first_id) {
    if (!w || (m && !records)) return fail(w, DYN_ERR_INVALID, "dyn_add_constraints: null argument");
    size_t before = w->joint_descs.size();
    for (uint32_t i = 0; i < m; ++i) {
        dyn_status st = add_constraint_record(w, records[i]);
        if (st) {  // all or nothing
            w->joint_descs.resize(before);
            w->joint_runtime.resize(before);
            return st;
        }
    }
    if (out_first_id) *out_first_id = (uint32_t)before;
    return DYN_OK;
}

// ---- body commands ----
DYN_API dyn_status dyn_edit_bodies(dyn_world* w, const uint32_t* body_ids, const dyn_body_edit_record* edits, uint32_t n) {
    if (!w || (n && (!body_ids || !edits))) return fail(w, DYN_ERR_INVALID, "dyn_edit_bodies: null argument");
    uint32_t ids = (uint32_t)std::max(w->spawn_states.size(), w->row_of_id.size());
    for (uint32_t i = 0; i < n; ++i) {
        if (body_ids[i] >= ids || (body_ids[i] < w->removed.size() && w->removed[body_ids[i]]))
            return fail(w, DYN_ERR_INVALID, "dyn_edit_bodies: unknown body id");
        if (edits[i].kind > DYN_EDIT_ANGULAR_IMPULSE) return fail(w, DYN_ERR_INVALID, "dyn_edit_bodies: unknown edit kind");
    }
    w->edit_ids.insert(w->edit_ids.end(), body_ids, body_ids + n);
    w->edits.insert(w->edits.end(), edits, edits + n);
    return DYN_OK;
}

// ---- removal ----
DYN_API dyn_status dyn_remove_bodies(dyn_world* w, const uint32_t* body_ids, uint32_t n) {
    if (!w || (n && !body_ids)) return fail(w, DYN_ERR_INVALID, "dyn_remove_bodies: null argument");
    if (w->raw_rows) return fail(w, DYN_ERR_INVALID, "dyn_remove_bodies: scene was replaced by dyn_upload_bodies");
    const uint32_t ids = (uint32_t)w->spawn_states.size();
    w->removed.resize(ids, 0u);
    std::vector<uint8_t> gone(ids, 0u);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t id = body_ids[i];
        if (id >= ids || w->removed[id] || gone[id]) return fail(w, DYN_ERR_INVALID, "dyn_remove_bodies: unknown or repeated body id");
        gone[id] = 1u;
    }
    // World::remove asserts the body is unreferenced (body.rs:132-134): a constraint still names it
    for (const dyn_constraint_descriptor_record& c : w->joint_descs) {
        if ((c.first_body_id < ids && gone[c.first_body_id]) || (c.second_body_id < ids && gone[c.second_body_id]))
            return fail(w, DYN_ERR_INVALID, "dyn_remove_bodies: a constraint still references the body");
    }
    if (dyn_status st = sync_spawn_states(w)) return st;  // the other bodies keep their simulated states
    for (uint32_t i = 0; i < n; ++i) w->removed[body_ids[i]] = 1u;
    w->rows_dirty = true;
    return DYN_OK;
}

// ---- batched worlds ----
DYN_API dyn_status dyn_set_body_worlds(dyn_world* w, const uint32_t* world_of_body, uint32_t n) {
    if (!w || (n && !world_of_body)) return fail(w, DYN_ERR_INVALID, "dyn_set_body_worlds: null argument");
    uint32_t ids = (uint32_t)std::max(w->spawn_states.size(), w->row_of_id.size());
    if (n != ids) return fail(w, DYN_ERR_INVALID, "dyn_set_body_worlds: one sub-world per body id");
    w->world_of_id.assign(world_of_body, world_of_body + n);
    if (w->raw_rows) {
        w->body_world.assign(w->states.size(), 0u);
        for (size_t r = 0; r < w->states.size(); ++r) {
            uint32_t id = w->states[r].body_id;
            if (id < n) w->body_world[r] = world_of_body[id];
        }
    } else {
        w->rows_dirty = true;
    }
    w->joints_dirty = true;
    if (w->dev) w->scene_dirty = true;
    return DYN_OK;
}

DYN_API dyn_status dyn_export_body_worlds(const dyn_world* cw, uint32_t* rows_out) {
    if (!cw || !rows_out) return DYN_ERR_INVALID;
    dyn_world* w = const_cast<dyn_world*>(cw);
    rebuild_rows(w);
    for (size_t r = 0; r < w->states.size(); ++r) rows_out[r] = r < w->body_world.size() ? w->body_world[r] : 0u;
    return DYN_OK;
}

DYN_API dyn_status dyn_constraint_count(const dyn_world* w, uint32_t* count) {
    if (!w || !count) return DYN_ERR_INVALID;
    *count = (uint32_t)w->joint_descs.size();
    return DYN_OK;
}

DYN_API dyn_status dyn_joint_plan(const dyn_world* cw, uint32_t* rows, uint32_t* layers, uint32_t* components,
                                  uint32_t* layer_count, uint32_t* component_count) {
    if (!cw) return DYN_ERR_INVALID;
    dyn_world* w = const_cast<dyn_world*>(cw);
    dyn_status st = rebuild_joints(w);
    if (st) return st;
    const JointPlan& p = w->joint_plan;
    if (rows) std::memcpy(rows, p.rows.data(), p.rows.size() * 4);
    if (layers) std::memcpy(layers, p.layers.data(), p.layers.size() * 4);
    if (components) std::memcpy(components, p.components.data(), p.components.size() * 4);
    if (layer_count) *layer_count = (uint32_t)(p.layers.size() / 2);
    if (component_count) *component_count = (uint32_t)(p.components.size() / 2);
    return DYN_OK;
}

DYN_API dyn_status dyn_export_constraints(const dyn_world* cw, dyn_constraint_descriptor_record* descs,
                                          dyn_constraint_rows_record* rows, dyn_constraint_runtime_record* runtime) {
    if (!cw) return DYN_ERR_INVALID;
    dyn_world* w = const_cast<dyn_world*>(cw);
    dyn_status st = rebuild_joints(w);
    if (st) return st;
    size_t m = w->joint_descs.size();
    if (descs) std::memcpy(descs, w->joint_descs.data(), m * sizeof(*descs));
    if (rows) std::memcpy(rows, w->joint_rows.data(), m * sizeof(*rows));
    if (runtime) std::memcpy(runtime, w->joint_runtime.data(), m * sizeof(*runtime));
    return DYN_OK;
}

}  // extern "C"
