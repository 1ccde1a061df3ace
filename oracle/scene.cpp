// oracle/scene.cpp - TEST INFRASTRUCTURE: the reference's scene set-up restated on the CPU, so that
// the oracle (and the reference arm of bench.py) can build a world's records without the product.
//
// Restates, from the reference:
//   PhysicsConfig::default                 crates/dynamis-model/src/config.rs:76-100
//   hull (add_hull_from_mesh)              crates/dynamis-hull/src/hull.rs:53-288
//   solid (hull mass integrals, f64)       crates/dynamis-hull/src/solid.rs:1-105
//   analytic_solid, compute_mass_properties, solid_volume_of, second_moment_*, inertia_inverse
//                                          crates/dynamis-model/src/mass.rs:1-330
//   quat_rotate                            crates/dynamis-model/src/math.rs:50-65
//   BodyStateRecord::initial, BodyDescriptorRecord::build
//                                          crates/dynamis-abi/src/body.rs:35-140
//   ColliderRecord::build, contact_relaxation
//                                          crates/dynamis-abi/src/collider.rs:8-103
//   ShapeScale::dimension_factor / record_scale and the shape roles
//                                          crates/dynamis-abi/src/shape.rs:48-193
//   the shape source record of a hull      crates/dynamis-world/src/shape_pool.rs:243-280,459-476,550-618
//   StepParamsRecord::new                  crates/dynamis-abi/src/param.rs:110-145
// and the row census the world uploads: dynamic rows (simulating, not kinematic) first, each group in
// body order. Bodies are given as the C ABI's dyn_body_desc / dyn_collider_desc (BodyDesc and
// ColliderDesc field for field); a hull source as a mesh (points and triangles), as
// add_hull_from_mesh takes it.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <vector>

#include "dynamis_abi.h"
#include "dynamis_cuda.h"

namespace {

using F3 = std::array<float, 3>;

F3 add(F3 a, F3 b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
F3 sub(F3 a, F3 b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
F3 mul(F3 v, float s) { return {v[0] * s, v[1] * s, v[2] * s}; }
float dot(F3 a, F3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
float length(F3 v) { return std::sqrt(dot(v, v)); }

// ---- hull.rs ----
struct Face {
    size_t a, b, c;
    F3 normal;
    float offset;
    std::vector<size_t> outside;
    bool dead = false;
};

F3 face_normal(const std::vector<F3>& p, size_t a, size_t b, size_t c) {
    const F3 ab = sub(p[b], p[a]), ac = sub(p[c], p[a]);
    const F3 cr = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
    const float len = length(cr);
    if (len < 1e-12f) return {0.0f, 0.0f, 0.0f};
    return {cr[0] / len, cr[1] / len, cr[2] / len};
}
Face make_face(const std::vector<F3>& p, size_t a, size_t b, size_t c) {
    Face f;
    f.a = a;
    f.b = b;
    f.c = c;
    f.normal = face_normal(p, a, b, c);
    f.offset = dot(f.normal, p[a]);
    return f;
}
float distance(const Face& f, F3 point) { return dot(f.normal, point) - f.offset; }

// assign_outside (hull.rs:194-208), except that a point which already is a corner of a face joins no
// outside set: rounding can put a corner beyond 1e-6 of a skinny face through it (near-duplicate
// points), and the reference's rounds then pick that corner again and again without end
void assign_outside(const std::vector<F3>& p, std::vector<Face>& faces, const std::vector<size_t>* restrict_to) {
    std::vector<uint8_t> corner(p.size(), 0);
    for (const Face& f : faces) corner[f.a] = corner[f.b] = corner[f.c] = 1;
    std::vector<size_t> candidates;
    if (restrict_to) {
        candidates = *restrict_to;
    } else {
        for (size_t i = 0; i < p.size(); ++i) candidates.push_back(i);
    }
    for (size_t point : candidates) {
        if (corner[point]) continue;
        for (Face& f : faces) {
            if (f.dead) continue;
            if (distance(f, p[point]) > 1e-6f) {
                f.outside.push_back(point);
                break;
            }
        }
    }
}

// Rust's max_by keeps the last of equal maxima; these do the same
bool quickhull(const std::vector<F3>& p, std::vector<size_t>* out_vertices, std::vector<std::array<size_t, 3>>* out_faces) {
    // extreme_pair
    size_t x_min = 0, x_max = 0;
    for (size_t i = 0; i < p.size(); ++i) {
        if (p[i][0] < p[x_min][0]) x_min = i;
        if (p[i][0] > p[x_max][0]) x_max = i;
    }
    size_t p0 = x_min, p1 = x_max;
    if (x_min == x_max) {
        p0 = 0;
        p1 = p.size() - 1;
    }
    // farthest_from_line
    const F3 dir = sub(p[p1], p[p0]);
    const float length_sq = dot(dir, dir);
    size_t p2 = 0;
    float best = -1.0f;
    for (size_t i = 0; i < p.size(); ++i) {
        const F3 delta = sub(p[i], p[p0]);
        const float projection = length_sq > 0.0f ? dot(delta, dir) / length_sq : 0.0f;
        const F3 closest = add(p[p0], mul(dir, projection));
        const float dist = length(sub(p[i], closest));
        if (dist > best) {
            best = dist;
            p2 = i;
        }
    }
    if (!(best > 1e-6f)) return false;  // collinear
    // farthest_from_plane
    const F3 plane_normal = face_normal(p, p0, p1, p2);
    const float plane_offset = dot(plane_normal, p[p0]);
    size_t p3 = 0;
    best = 0.0f;
    for (size_t i = 0; i < p.size(); ++i) {
        const float dist = std::fabs(dot(plane_normal, p[i]) - plane_offset);
        if (dist > best) {
            best = dist;
            p3 = i;
        }
    }
    if (!(best > 1e-6f)) return false;  // coplanar
    // initial_tetra
    F3 centroid;
    for (int a = 0; a < 3; ++a) centroid[a] = (p[p0][a] + p[p1][a] + p[p2][a] + p[p3][a]) * 0.25f;
    std::vector<Face> faces = {make_face(p, p0, p1, p2), make_face(p, p0, p1, p3), make_face(p, p0, p2, p3),
                               make_face(p, p1, p2, p3)};
    for (Face& f : faces) {
        if (dot(f.normal, centroid) - f.offset > 0.0f) {
            f.normal = {-f.normal[0], -f.normal[1], -f.normal[2]};
            f.offset = -f.offset;
            std::swap(f.b, f.c);
        }
    }
    assign_outside(p, faces, nullptr);
    std::vector<size_t> indices;
    for (size_t i = 0; i < faces.size(); ++i) indices.push_back(i);
    while (!indices.empty()) {
        std::vector<size_t> kept;
        for (size_t i : indices)
            if (!faces[i].dead && !faces[i].outside.empty()) kept.push_back(i);
        indices = kept;
        if (indices.empty()) break;
        size_t seed = indices[0];
        float seed_key = distance(faces[seed], p[faces[seed].outside.front()]);
        for (size_t k = 1; k < indices.size(); ++k) {
            const float key = distance(faces[indices[k]], p[faces[indices[k]].outside.front()]);
            if (!(key < seed_key)) {
                seed = indices[k];
                seed_key = key;
            }
        }
        const Face& sf = faces[seed];
        size_t apex = sf.outside[0];
        float apex_key = distance(sf, p[apex]);
        for (size_t k = 1; k < sf.outside.size(); ++k) {
            const float key = distance(sf, p[sf.outside[k]]);
            if (!(key < apex_key)) {
                apex = sf.outside[k];
                apex_key = key;
            }
        }
        std::vector<size_t> visible;
        for (size_t i = 0; i < faces.size(); ++i)
            if (!faces[i].dead && i != seed && distance(faces[i], p[apex]) > 1e-6f) visible.push_back(i);
        visible.push_back(seed);
        std::set<std::pair<size_t, size_t>> edges;
        for (size_t i : visible) {
            const Face& f = faces[i];
            edges.insert({f.a, f.b});
            edges.insert({f.b, f.c});
            edges.insert({f.c, f.a});
        }
        std::vector<std::pair<size_t, size_t>> horizon;
        for (size_t i : visible) {
            const Face& f = faces[i];
            const std::pair<size_t, size_t> es[3] = {{f.a, f.b}, {f.b, f.c}, {f.c, f.a}};
            for (const auto& e : es)
                if (!edges.count({e.second, e.first})) horizon.push_back(e);
        }
        if (horizon.empty()) return false;
        std::vector<size_t> pending;
        for (size_t i : visible) {
            pending.insert(pending.end(), faces[i].outside.begin(), faces[i].outside.end());
            faces[i].dead = true;
        }
        pending.push_back(apex);
        for (const auto& e : horizon) faces.push_back(make_face(p, e.first, e.second, apex));
        assign_outside(p, faces, &pending);
        indices.clear();
        for (size_t i = 0; i < faces.size(); ++i) indices.push_back(i);
    }
    out_faces->clear();
    out_vertices->clear();
    for (const Face& f : faces) {
        if (f.dead) continue;
        out_faces->push_back({f.a, f.b, f.c});
        for (size_t v : {f.a, f.b, f.c})
            if (std::find(out_vertices->begin(), out_vertices->end(), v) == out_vertices->end()) out_vertices->push_back(v);
    }
    return true;
}

struct HullSource {
    std::vector<F3> vertices;
    std::vector<std::array<uint32_t, 3>> triangles;
    float volume = 0.0f;
    F3 centroid{};
    float unit_second[6]{};
};

// hull(): the points the triangles reference, in ascending index order, hulled; vertices in first
// appearance over the surviving faces
bool hull_of_mesh(const float* xyz, uint32_t nv, const uint32_t* tris, uint32_t nt, HullSource* h) {
    std::set<uint32_t> used;
    for (uint32_t t = 0; t < 3 * nt; ++t) {
        if (tris[t] >= nv) return false;
        used.insert(tris[t]);
    }
    std::vector<F3> points;
    for (uint32_t i : used) points.push_back({xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]});
    std::vector<size_t> order;
    std::vector<std::array<size_t, 3>> faces;
    if (points.size() < 4 || !quickhull(points, &order, &faces)) return false;
    std::map<size_t, uint32_t> remap;
    for (size_t v : order) {
        if (remap.count(v)) continue;
        remap[v] = (uint32_t)h->vertices.size();
        h->vertices.push_back(points[v]);
    }
    for (const auto& f : faces) h->triangles.push_back({remap[f[0]], remap[f[1]], remap[f[2]]});
    return true;
}

// ---- solid.rs (f64) ----
using D3 = std::array<double, 3>;
D3 dcross(D3 a, D3 b) { return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}; }
double ddot(D3 a, D3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

bool hull_solid(HullSource* h) {
    double sum[3] = {0.0, 0.0, 0.0};
    for (const F3& v : h->vertices)
        for (int a = 0; a < 3; ++a) sum[a] += (double)v[a];
    const double count = (double)h->vertices.size();
    const D3 apex = {sum[0] / count, sum[1] / count, sum[2] / count};
    auto shifted = [&](const F3& v) { return D3{(double)v[0] - apex[0], (double)v[1] - apex[1], (double)v[2] - apex[2]}; };
    auto squared = [](double ax, double bx, double cx) { return (ax * ax + bx * bx + cx * cx + ax * bx + ax * cx + bx * cx) / 10.0; };
    auto mixed = [](double ax, double bx, double cx, double ay, double by, double cy) {
        return (2.0 * (ax * ay + bx * by + cx * cy) + ax * by + ay * bx + ax * cy + ay * cx + bx * cy + by * cx) / 20.0;
    };
    double volume = 0.0, first[3] = {0.0, 0.0, 0.0}, second[6] = {0, 0, 0, 0, 0, 0};
    for (const auto& t : h->triangles) {
        D3 a = shifted(h->vertices[t[0]]), b = shifted(h->vertices[t[1]]), c = shifted(h->vertices[t[2]]);
        if (ddot(dcross(a, b), c) < 0.0) std::swap(b, c);
        const double s = ddot(a, dcross(b, c)) / 6.0;
        volume += s;
        for (int k = 0; k < 3; ++k) first[k] += s * (a[k] + b[k] + c[k]) / 4.0;
        second[0] += s * squared(a[0], b[0], c[0]);
        second[3] += s * squared(a[1], b[1], c[1]);
        second[5] += s * squared(a[2], b[2], c[2]);
        second[1] += s * mixed(a[0], b[0], c[0], a[1], b[1], c[1]);
        second[2] += s * mixed(a[0], b[0], c[0], a[2], b[2], c[2]);
        second[4] += s * mixed(a[1], b[1], c[1], a[2], b[2], c[2]);
    }
    if (!(volume > 0.0) || !std::isfinite(volume)) return false;
    const double cen[3] = {first[0] / volume, first[1] / volume, first[2] / volume};
    h->volume = (float)volume;
    for (int k = 0; k < 3; ++k) h->centroid[k] = (float)(apex[k] + cen[k]);
    const int ij[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    for (int q = 0; q < 6; ++q)
        h->unit_second[q] = (float)((second[q] - volume * cen[ij[q][0]] * cen[ij[q][1]]) / volume);
    return true;
}

// ---- mass.rs ----
struct Solid {
    float volume;
    F3 centroid;
    float second[6];
};

F3 quat_rotate(const float q[4], F3 v) {
    const F3 u = {q[0], q[1], q[2]};
    const float s = q[3];
    const float d = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
    const float square = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const F3 c = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    F3 out;
    for (int a = 0; a < 3; ++a) out[a] = v[a] + 2.0f * (s * c[a] + d * u[a] - square * v[a]);
    return out;
}

bool analytic_solid(const dyn_collider_desc& c, const std::vector<HullSource>& hulls, Solid* s) {
    const float pi = 3.14159265358979323846f;
    std::memset(s, 0, sizeof(*s));
    switch (c.shape) {
        case DYN_SHAPE_SPHERE: {
            const float r = c.radius, moment = r * r / 5.0f;
            s->volume = 4.0f / 3.0f * pi * r * r * r;
            s->second[0] = s->second[3] = s->second[5] = moment;
            return true;
        }
        case DYN_SHAPE_CUBOID: {
            const float ex = c.half_extents[0] * 2.0f, ey = c.half_extents[1] * 2.0f, ez = c.half_extents[2] * 2.0f;
            s->volume = ex * ey * ez;
            s->second[0] = ex * ex / 12.0f;
            s->second[3] = ey * ey / 12.0f;
            s->second[5] = ez * ez / 12.0f;
            return true;
        }
        case DYN_SHAPE_CAPSULE: {
            const float r = c.radius, hh = c.half_height;
            const float cylinder = pi * r * r * 2.0f * hh;
            const float sphere = 4.0f / 3.0f * pi * r * r * r;
            const float total = cylinder + sphere;
            const float lateral = (cylinder * r * r / 4.0f + sphere * r * r / 5.0f) / total;
            const float axial = (cylinder * 4.0f * hh * hh / 12.0f + sphere * (r * r / 5.0f + 3.0f / 4.0f * r * hh + hh * hh)) / total;
            s->volume = total;
            s->second[0] = lateral;
            s->second[3] = axial;
            s->second[5] = lateral;
            return true;
        }
        case DYN_SHAPE_CYLINDER: {
            const float r = c.radius, height = c.half_height * 2.0f, lateral = r * r / 4.0f;
            s->volume = pi * r * r * height;
            s->second[0] = lateral;
            s->second[3] = height * height / 12.0f;
            s->second[5] = lateral;
            return true;
        }
        case DYN_SHAPE_HULL: {
            if (c.source >= hulls.size()) return false;
            const HullSource& h = hulls[c.source];
            s->volume = h.volume;
            s->centroid = h.centroid;
            for (int q = 0; q < 6; ++q) s->second[q] = h.unit_second[q];
            return true;
        }
        default:
            return false;
    }
}

F3 centroid_of(const dyn_collider_desc& c, const Solid& s) {
    const F3 scaled = {c.scale[0] * s.centroid[0], c.scale[1] * s.centroid[1], c.scale[2] * s.centroid[2]};
    const F3 rotated = quat_rotate(c.rotation, scaled);
    return {c.offset[0] + rotated[0], c.offset[1] + rotated[1], c.offset[2] + rotated[2]};
}

using M3 = std::array<std::array<float, 3>, 3>;
M3 mat_from_quat(const float q[4]) {
    const float x = q[0], y = q[1], z = q[2], w = q[3];
    return M3{{{1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y - w * z), 2.0f * (x * z + w * y)},
               {2.0f * (x * y + w * z), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z - w * x)},
               {2.0f * (x * z - w * y), 2.0f * (y * z + w * x), 1.0f - 2.0f * (x * x + y * y)}}};
}
M3 mat_mul(const M3& a, const M3& b) {
    M3 r{};
    for (int row = 0; row < 3; ++row)
        for (int col = 0; col < 3; ++col) r[row][col] = a[row][0] * b[0][col] + a[row][1] * b[1][col] + a[row][2] * b[2][col];
    return r;
}

struct MassProperties {
    F3 com{};
    float inertia[6]{};
    float inverse_inertia[6]{};
};

bool inertia_inverse(const float in[6], float out[6]) {
    const float xx = in[0], xy = in[1], xz = in[2], yy = in[3], yz = in[4], zz = in[5];
    const float cxx = yy * zz - yz * yz, cxy = xz * yz - xy * zz, cxz = xy * yz - xz * yy;
    const float cyy = xx * zz - xz * xz, cyz = xy * xz - xx * yz, czz = xx * yy - xy * xy;
    const float det = xx * cxx + xy * cxy + xz * cxz;
    if (!(xx > 0.0f && czz > 0.0f && det > 0.0f)) return false;
    const float cof[6] = {cxx, cxy, cxz, cyy, cyz, czz};
    for (int q = 0; q < 6; ++q) out[q] = cof[q] / det;
    return true;
}

// compute_mass_properties with MassSource::Density(density) or ::Fixed(mass); no com override
bool mass_properties(const dyn_collider_desc* cols, uint32_t count, const std::vector<HullSource>& hulls, bool density_mode,
                     float amount, MassProperties* out) {
    *out = MassProperties{};
    std::vector<const dyn_collider_desc*> which;
    std::vector<Solid> solids;
    for (uint32_t c = 0; c < count; ++c) {
        if (cols[c].sensor) continue;
        Solid s;
        if (!analytic_solid(cols[c], hulls, &s)) continue;
        which.push_back(&cols[c]);
        solids.push_back(s);
    }
    if (solids.empty()) return true;
    std::vector<float> volumes;
    float total = 0.0f;
    for (size_t i = 0; i < solids.size(); ++i) {
        volumes.push_back(which[i]->scale[0] * which[i]->scale[1] * which[i]->scale[2] * solids[i].volume);
        total += volumes.back();
    }
    if (total <= 0.0f) return true;
    const float mass = density_mode ? amount * total : amount;
    if (mass <= 0.0f) return true;
    F3 sum = {0.0f, 0.0f, 0.0f};
    for (size_t i = 0; i < solids.size(); ++i) {
        const F3 at = centroid_of(*which[i], solids[i]);
        for (int a = 0; a < 3; ++a) sum[a] += at[a] * volumes[i];
    }
    const F3 com = {sum[0] / total, sum[1] / total, sum[2] / total};
    float second[6] = {0, 0, 0, 0, 0, 0};
    for (size_t i = 0; i < solids.size(); ++i) {
        const dyn_collider_desc& c = *which[i];
        const float shape_mass = mass * volumes[i] / total;
        const float* u = solids[i].second;
        const float* sc = c.scale;
        const float local[6] = {u[0] * sc[0] * sc[0], u[1] * sc[0] * sc[1], u[2] * sc[0] * sc[2],
                                u[3] * sc[1] * sc[1], u[4] * sc[1] * sc[2], u[5] * sc[2] * sc[2]};
        const M3 r = mat_from_quat(c.rotation);
        const M3 sm = {{{local[0], local[1], local[2]}, {local[1], local[3], local[4]}, {local[2], local[4], local[5]}}};
        const M3 rt = {{{r[0][0], r[1][0], r[2][0]}, {r[0][1], r[1][1], r[2][1]}, {r[0][2], r[1][2], r[2][2]}}};
        const M3 m = mat_mul(r, mat_mul(sm, rt));
        const float rotated[6] = {m[0][0], (m[0][1] + m[1][0]) * 0.5f, (m[0][2] + m[2][0]) * 0.5f,
                                  m[1][1], (m[1][2] + m[2][1]) * 0.5f, m[2][2]};
        const F3 at = centroid_of(c, solids[i]);
        const F3 d = {at[0] - com[0], at[1] - com[1], at[2] - com[2]};
        const float translated[6] = {rotated[0] + d[0] * d[0], rotated[1] + d[0] * d[1], rotated[2] + d[0] * d[2],
                                     rotated[3] + d[1] * d[1], rotated[4] + d[1] * d[2], rotated[5] + d[2] * d[2]};
        for (int q = 0; q < 6; ++q) second[q] += translated[q] * shape_mass;
    }
    const float xx = second[0], xy = second[1], xz = second[2], yy = second[3], yz = second[4], zz = second[5];
    const float inertia[6] = {yy + zz, -xy, -xz, xx + zz, -yz, xx + yy};
    out->com = com;
    for (int q = 0; q < 6; ++q) out->inertia[q] = inertia[q];
    return inertia_inverse(inertia, out->inverse_inertia);
}

float solid_volume_of(const dyn_collider_desc* cols, uint32_t count, const std::vector<HullSource>& hulls) {
    float total = 0.0f;
    for (uint32_t c = 0; c < count; ++c) {
        if (cols[c].sensor) continue;
        Solid s;
        if (!analytic_solid(cols[c], hulls, &s)) continue;
        total += cols[c].scale[0] * cols[c].scale[1] * cols[c].scale[2] * s.volume;
    }
    return total;
}

// ---- abi collider.rs / shape.rs ----
enum class Scale { NotScalable, UniformFolded, InDimensions, InRecord };
Scale scale_rule(uint32_t shape) {
    switch (shape) {
        case DYN_SHAPE_SPHERE:
        case DYN_SHAPE_CAPSULE:
        case DYN_SHAPE_CYLINDER: return Scale::UniformFolded;
        case DYN_SHAPE_CUBOID: return Scale::InDimensions;
        case DYN_SHAPE_HULL: return Scale::InRecord;
        default: return Scale::NotScalable;
    }
}
bool uniform(const float s[3]) { return s[0] == s[1] && s[1] == s[2]; }

dyn_collider_record collider_record(const dyn_collider_desc& c, uint32_t slot) {
    dyn_collider_record r;
    std::memset(&r, 0, sizeof(r));
    const Scale rule = scale_rule(c.shape);
    float factor[3] = {1.0f, 1.0f, 1.0f};
    if (rule == Scale::InDimensions) {
        for (int a = 0; a < 3; ++a) factor[a] = c.scale[a];
    } else if (rule == Scale::UniformFolded && uniform(c.scale)) {
        for (int a = 0; a < 3; ++a) factor[a] = c.scale[0];
    }
    uint32_t flags = c.sensor ? DYN_COLLIDER_SENSOR : 0u;
    if (c.events & DYN_EVENT_MODE_PERSIST) {
        flags |= DYN_EVENT_MODE_BEGIN_END | DYN_EVENT_MODE_PERSIST;
    } else if (c.events & DYN_EVENT_MODE_BEGIN_END) {
        flags |= DYN_EVENT_MODE_BEGIN_END;
    }
    r.slot = slot;
    r.kind = c.shape;
    r.flags = flags;
    const bool round = c.shape == DYN_SHAPE_SPHERE || c.shape == DYN_SHAPE_CAPSULE || c.shape == DYN_SHAPE_CYLINDER;
    r.radius = round ? c.radius * factor[0] : 0.0f;
    r.half_height = (c.shape == DYN_SHAPE_CAPSULE || c.shape == DYN_SHAPE_CYLINDER) ? c.half_height * factor[0] : 0.0f;
    r.impact_force = c.impact_force;
    if (c.shape == DYN_SHAPE_CUBOID)
        for (int a = 0; a < 3; ++a) r.half_extents[a] = c.half_extents[a] * factor[a];
    r.collision_group = c.collision_group;
    r.collision_mask = c.collision_mask;
    for (int a = 0; a < 3; ++a) r.local_offset[a] = c.offset[a];
    for (int a = 0; a < 4; ++a) r.local_rotation[a] = c.rotation[a];
    r.friction = c.friction;
    r.restitution = c.restitution;
    r.source = c.shape == DYN_SHAPE_HULL ? c.source : 0u;
    r.rolling_friction = c.rolling_friction;
    const bool keep = rule == Scale::InRecord || (rule == Scale::UniformFolded && !uniform(c.scale));
    for (int a = 0; a < 3; ++a) r.scale[a] = keep ? c.scale[a] : 1.0f;
    r.spin_friction = c.spin_friction;
    r.relaxation = std::isinf(c.contact_frequency) ? 0.0f : 1.0f / (6.28318530717958647692f * c.contact_frequency);
    r.damping_ratio = c.contact_damping_ratio;
    return r;
}

}  // namespace

struct OrcScene {
    dyn_config config;
    std::vector<HullSource> hulls;
    std::vector<dyn_body_state_record> states;
    std::vector<dyn_body_descriptor_record> descs;
    std::vector<dyn_collider_record> colliders;
    std::vector<uint32_t> owners;
    uint32_t dynamic_count = 0;
    int error = 0;  // 0, or the index + 1 of the first body (or -(hull + 1)) that could not be built
};

extern "C" {

// PhysicsConfig::default
void orc_config_default(dyn_config* c) {
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

// A hull source from a mesh (add_hull_from_mesh): returns its vertex count, or 0 when the mesh
// spans no volume or a triangle names a vertex outside it. Out may be null (count only); else it
// receives the hull's vertices (3 floats each, in dynamis-hull's order) and, when tris_out is not
// null, its triangles (up to tris_cap).
uint32_t orc_hull_from_mesh(const float* xyz, uint32_t nv, const uint32_t* tris, uint32_t nt, float* out, uint32_t* tris_out,
                            uint32_t tris_cap, uint32_t* tri_count) {
    HullSource h;
    if (!hull_of_mesh(xyz, nv, tris, nt, &h)) return 0;
    if (out)
        for (size_t i = 0; i < h.vertices.size(); ++i)
            for (int a = 0; a < 3; ++a) out[3 * i + a] = h.vertices[i][a];
    if (tri_count) *tri_count = (uint32_t)h.triangles.size();
    if (tris_out)
        for (size_t t = 0; t < h.triangles.size() && t < tris_cap; ++t)
            for (int a = 0; a < 3; ++a) tris_out[3 * t + a] = h.triangles[t][a];
    return (uint32_t)h.vertices.size();
}

// Builds a scene's records as the reference's World::spawn and its upload would: hull sources
// first (hull_first[s] .. hull_first[s + 1] index points, tri_first likewise triangles; a null
// tris means every point is referenced), then the bodies in order. config null = the defaults.
OrcScene* orc_scene_build(const dyn_config* config, const float* hull_points, const uint32_t* hull_first, const uint32_t* tris,
                          const uint32_t* tri_first, uint32_t hulls, const dyn_body_desc* bodies, uint32_t n,
                          const dyn_collider_desc* cols, uint32_t k) {
    OrcScene* s = new OrcScene();
    if (config) {
        s->config = *config;
    } else {
        orc_config_default(&s->config);
    }
    for (uint32_t h = 0; h < hulls; ++h) {
        const uint32_t first = hull_first[h], count = hull_first[h + 1] - first;
        std::vector<uint32_t> all;
        const uint32_t* t = nullptr;
        uint32_t nt = 0;
        if (tris) {
            t = tris + 3 * (size_t)tri_first[h];
            nt = tri_first[h + 1] - tri_first[h];
        } else {
            for (uint32_t i = 0; i < count; ++i) all.push_back(i);
            while (all.size() % 3) all.push_back(count - 1);
            t = all.data();
            nt = (uint32_t)all.size() / 3;
        }
        HullSource src;
        if (!hull_of_mesh(hull_points + 3 * (size_t)first, count, t, nt, &src) || !hull_solid(&src)) {
            s->error = -(int)(h + 1);
            return s;
        }
        s->hulls.push_back(std::move(src));
    }
    std::vector<dyn_body_state_record> spawn_states;
    std::vector<dyn_body_descriptor_record> spawn_descs;
    std::vector<dyn_collider_record> spawn_colliders;
    std::vector<uint32_t> spawn_owner;
    for (uint32_t b = 0; b < n; ++b) {
        const dyn_body_desc& bd = bodies[b];
        if (bd.collider_count == 0 || (uint64_t)bd.collider_first + bd.collider_count > k) {
            s->error = (int)b + 1;
            return s;
        }
        const dyn_collider_desc* bc = cols + bd.collider_first;
        // BodyDesc::effective_mass / kind: density x solid volume, or the given mass
        const bool density_mode = bd.density > 0.0f;
        const float mass = density_mode ? bd.density * solid_volume_of(bc, bd.collider_count, s->hulls) : bd.mass;
        const bool simulates = !bd.kinematic && mass > 0.0f;
        MassProperties props;
        if (!mass_properties(bc, bd.collider_count, s->hulls, density_mode, density_mode ? bd.density : bd.mass, &props)) {
            s->error = (int)b + 1;
            return s;
        }
        dyn_body_descriptor_record d;
        std::memset(&d, 0, sizeof(d));
        d.inverse_mass = simulates ? 1.0f / mass : 0.0f;
        d.linear_damping = bd.linear_damping >= 0.0f ? bd.linear_damping : s->config.damping;
        d.angular_damping = bd.angular_damping >= 0.0f ? bd.angular_damping : s->config.angular_damping;
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
        for (int a = 0; a < 3; ++a) d.com[a] = props.com[a];
        for (int q = 0; q < 6; ++q) {
            d.inertia[q] = props.inertia[q];
            d.inverse_inertia[q] = props.inverse_inertia[q];
        }
        dyn_body_state_record st;
        std::memset(&st, 0, sizeof(st));
        for (int a = 0; a < 3; ++a) {
            st.position[a] = bd.position[a];
            st.prev_position[a] = bd.position[a];
            st.velocity[a] = bd.velocity[a];
            st.angular_velocity[a] = bd.angular_velocity[a];
        }
        for (int a = 0; a < 4; ++a) {
            st.orientation[a] = bd.orientation[a];
            st.prev_orientation[a] = bd.orientation[a];
        }
        st.body_id = b;
        spawn_states.push_back(st);
        spawn_descs.push_back(d);
        for (uint32_t c = 0; c < bd.collider_count; ++c) {
            spawn_colliders.push_back(collider_record(bc[c], (uint32_t)spawn_colliders.size()));
            spawn_owner.push_back(b);
        }
    }
    // the row census: simulating (non-kinematic, positive inverse mass) rows first
    std::vector<uint32_t> order, row_of(n, 0);
    for (uint32_t pass = 0; pass < 2; ++pass)
        for (uint32_t i = 0; i < n; ++i) {
            const bool dyn = (spawn_descs[i].flags & DYN_BODY_KINEMATIC) == 0u && spawn_descs[i].inverse_mass > 0.0f;
            if (dyn == (pass == 0)) order.push_back(i);
        }
    for (uint32_t i = 0; i < n; ++i) {
        const dyn_body_descriptor_record& d = spawn_descs[i];
        if ((d.flags & DYN_BODY_KINEMATIC) == 0u && d.inverse_mass > 0.0f) s->dynamic_count += 1;
    }
    for (uint32_t r = 0; r < n; ++r) {
        s->states.push_back(spawn_states[order[r]]);
        s->descs.push_back(spawn_descs[order[r]]);
        row_of[order[r]] = r;
    }
    s->colliders = spawn_colliders;
    for (uint32_t o : spawn_owner) s->owners.push_back(row_of[o]);
    return s;
}

int orc_scene_error(const OrcScene* s) { return s->error; }
void orc_scene_free(OrcScene* s) { delete s; }

void orc_scene_sizes(const OrcScene* s, uint32_t* bodies, uint32_t* dynamic, uint32_t* colliders, uint32_t* sources,
                     uint32_t* vertices) {
    *bodies = (uint32_t)s->states.size();
    *dynamic = s->dynamic_count;
    *colliders = (uint32_t)s->colliders.size();
    *sources = (uint32_t)s->hulls.size();
    uint32_t v = 0;
    for (const HullSource& h : s->hulls) v += (uint32_t)h.vertices.size();
    *vertices = v;
}

// The records, with the hull sources as the shape pool lays them out: vertex rows (x, y, z, 0) one
// source after another, each source's local bounds over its vertices.
void orc_scene_export(const OrcScene* s, dyn_body_state_record* states, dyn_body_descriptor_record* descs,
                      dyn_collider_record* colliders, uint32_t* owners, dyn_shape_source_record* sources, float* vertices) {
    std::copy(s->states.begin(), s->states.end(), states);
    std::copy(s->descs.begin(), s->descs.end(), descs);
    std::copy(s->colliders.begin(), s->colliders.end(), colliders);
    std::copy(s->owners.begin(), s->owners.end(), owners);
    uint32_t offset = 0;
    for (size_t h = 0; h < s->hulls.size(); ++h) {
        const HullSource& src = s->hulls[h];
        dyn_shape_source_record& r = sources[h];
        std::memset(&r, 0, sizeof(r));
        r.kind = DYN_SHAPE_HULL;
        r.vertex_offset = offset;
        r.vertex_count = (uint32_t)src.vertices.size();
        float lo[3] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
        float hi[3] = {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
        for (const F3& v : src.vertices) {
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], v[a]);
                hi[a] = std::max(hi[a], v[a]);
                vertices[4 * (size_t)offset + a] = v[a];
            }
            vertices[4 * (size_t)offset + 3] = 0.0f;
            ++offset;
        }
        for (int a = 0; a < 3; ++a) {
            r.local_min[a] = lo[a];
            r.local_max[a] = hi[a];
        }
    }
}

// StepParamsRecord::new for this scene's census (no joints, soft bodies or observations)
void orc_scene_params(const OrcScene* s, float dt, dyn_step_params* out) {
    const dyn_config& c = s->config;
    std::memset(out, 0, sizeof(*out));
    for (int a = 0; a < 3; ++a) out->gravity[a] = c.gravity[a];
    out->dt = dt;
    out->substep_dt = dt / (float)c.substeps;
    out->damping = c.damping;
    out->angular_damping = c.angular_damping;
    out->body_count = (uint32_t)s->states.size();
    out->substeps = c.substeps;
    out->solve_iterations = c.solve_iterations;
    out->relaxation = c.relaxation;
    out->slop = c.slop;
    out->restitution_threshold = c.restitution_threshold;
    out->max_velocity = c.max_velocity;
    out->max_angular_velocity = c.max_angular_velocity;
    out->dynamic_count = s->dynamic_count;
    out->sleep_velocity = c.sleep_velocity;
    out->sleep_angular_velocity = c.sleep_angular_velocity;
    out->sleep_time = c.sleep_time;
    out->friction_combine = c.friction_combine;
    out->restitution_combine = c.restitution_combine;
    out->position_iterations = c.position_iterations;
    out->contact_margin = c.contact_margin;
    out->collider_count = (uint32_t)s->colliders.size();
    out->soft_iterations = 1;
    out->soft_substeps = 4;
    out->soft_substep_dt = dt / 4.0f;
    out->settle_velocity = 1.0e-4f;
}

}  // extern "C"
