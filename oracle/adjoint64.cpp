// adjoint64.cpp - FP64 reference for the differentiable step over a frozen contact set.
//
// TEST INFRASTRUCTURE ONLY (loaded by tests/ and bench.py's checks through oracle/adjoint.py; the
// product never links it). It restates, in double precision, the part of World::step that the
// adjoint differentiates: substep integration (substep_integrate.wgsl:15-76), the contact solve
// (solver_contact_block.wgsl:6-233 with core.wgsl:326-345; target speeds of solver_blocks.wgsl:24-48),
// advance (substep_advance.wgsl:6-13) and position correction (position_correction.wgsl:5-46,
// position_block.wgsl:11-33, position_apply.wgsl:12-27), stepping over contact sets given per step:
// the contacts, their local anchors, normals, narrowphase depths and relay sources are inputs, not
// recomputed. The fixed-point delta accumulation of the device (core.wgsl:6-12) is replaced by
// exact sums, the solver's order-independent intent.
//
// The depth a step's solve and position passes read is the narrowphase depth at the step's start,
// d = d0 + n . ((x_a + R_a la) - (x_b + R_b lb)), with la, lb the point's anchors in each body's
// frame (both at the contact point when the narrowphase ran, so d = d0 on the recorded poses): the
// depth of the frozen contact moves with the bodies to first order.
//
// Everything is a template on the scalar type: double gives the FP64 forward whose central
// differences the gradient checks use; Dual<K> (forward-mode derivatives along K directions of the
// parameter space) gives the reference gradient the device adjoint is checked against.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace adj {

// ---- forward-mode dual numbers ----
template <int K>
struct Dual {
    double v = 0.0;
    double d[K] = {};
    Dual() = default;
    Dual(double x) : v(x) {}  // NOLINT: constants promote implicitly
};
template <int K> Dual<K> operator+(const Dual<K>& a, const Dual<K>& b) { Dual<K> r(a.v + b.v); for (int i = 0; i < K; ++i) r.d[i] = a.d[i] + b.d[i]; return r; }
template <int K> Dual<K> operator-(const Dual<K>& a, const Dual<K>& b) { Dual<K> r(a.v - b.v); for (int i = 0; i < K; ++i) r.d[i] = a.d[i] - b.d[i]; return r; }
template <int K> Dual<K> operator-(const Dual<K>& a) { Dual<K> r(-a.v); for (int i = 0; i < K; ++i) r.d[i] = -a.d[i]; return r; }
template <int K> Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) { Dual<K> r(a.v * b.v); for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r; }
template <int K> Dual<K> operator/(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r(a.v / b.v);
    for (int i = 0; i < K; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
    return r;
}
template <int K> Dual<K> sqrt(const Dual<K>& a) {
    Dual<K> r(std::sqrt(a.v));
    for (int i = 0; i < K; ++i) r.d[i] = r.v > 0.0 ? a.d[i] / (2.0 * r.v) : 0.0;
    return r;
}
template <int K> Dual<K> sin(const Dual<K>& a) { Dual<K> r(std::sin(a.v)); double c = std::cos(a.v); for (int i = 0; i < K; ++i) r.d[i] = c * a.d[i]; return r; }
template <int K> Dual<K> cos(const Dual<K>& a) { Dual<K> r(std::cos(a.v)); double s = -std::sin(a.v); for (int i = 0; i < K; ++i) r.d[i] = s * a.d[i]; return r; }
template <int K> Dual<K>& operator+=(Dual<K>& a, const Dual<K>& b) { a = a + b; return a; }
inline double val(double x) { return x; }
template <int K> double val(const Dual<K>& x) { return x.v; }
using std::sqrt;
using std::sin;
using std::cos;

// ---- vectors and quaternions (core.wgsl:132-178, 347-394) ----
template <class T> struct V3 { T x, y, z; };
template <class T> struct Q4 { T x, y, z, w; };
template <class T> V3<T> operator+(const V3<T>& a, const V3<T>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> V3<T> operator-(const V3<T>& a, const V3<T>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> V3<T> operator-(const V3<T>& a) { return {-a.x, -a.y, -a.z}; }
template <class T> V3<T> operator*(const V3<T>& a, const T& s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> V3<T> operator/(const V3<T>& a, const T& s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> T dot(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> V3<T> cross(const V3<T>& a, const V3<T>& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> T length(const V3<T>& a) { return sqrt(dot(a, a)); }
template <class T> V3<T> zero3() { return {T(0.0), T(0.0), T(0.0)}; }
template <class T> Q4<T> quat_mul(const Q4<T>& a, const Q4<T>& b) {
    V3<T> av{a.x, a.y, a.z}, bv{b.x, b.y, b.z};
    V3<T> v = bv * a.w + av * b.w + cross(av, bv);
    return {v.x, v.y, v.z, a.w * b.w - dot(av, bv)};
}
template <class T> Q4<T> quat_conj(const Q4<T>& q) { return {-q.x, -q.y, -q.z, q.w}; }
template <class T> V3<T> quat_rotate(const Q4<T>& q, const V3<T>& v) {
    V3<T> u{q.x, q.y, q.z};
    return u * (T(2.0) * dot(u, v)) + v * (q.w * q.w - dot(u, u)) + cross(u, v) * (T(2.0) * q.w);
}
template <class T> Q4<T> normalize4(const Q4<T>& q) {
    T n = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    return {q.x / n, q.y / n, q.z / n, q.w / n};
}
template <class T> V3<T> sym_apply(const T* t, const V3<T>& v) {
    return {t[0] * v.x + t[1] * v.y + t[2] * v.z, t[1] * v.x + t[3] * v.y + t[4] * v.z, t[2] * v.x + t[4] * v.y + t[5] * v.z};
}
template <class T> V3<T> rotate_about(const V3<T>& rotation, const V3<T>& v) {
    T angle = length(rotation);
    if (val(angle) < 1e-8) return v;
    V3<T> axis = rotation / angle;
    V3<T> offset = cross(axis, v);
    return v + offset * sin(angle) + cross(axis, offset) * (T(1.0) - cos(angle));
}
template <class T> T wmax(const T& a, const T& b) { return val(a) > val(b) ? a : b; }
template <class T> T wclamp(const T& x, const T& lo, const T& hi) {
    T m = val(x) > val(lo) ? x : lo;
    return val(m) < val(hi) ? m : hi;
}

// ---- the frozen problem ----
struct Params {
    double dt, gravity[3], slop, relaxation, restitution_threshold, max_velocity, max_angular_velocity;
    uint32_t substeps, iterations, position_iterations;
};
struct BodyConst {
    double com[3], gravity_scale, linear_damping, angular_damping, inertia[6];
    bool dynamic;  // simulated and awake: integrated, solved and corrected
};
struct ContactIn {
    uint32_t a, b, count, group;
    bool resolves;
    double normal[3], restitution, rolling, spin, relaxation, damping_ratio;
    double la[4][3], lb[4][3], depth[4], position[4][3], acc[4][3];
    int32_t source[4];  // index of the relayed point in the previous step's points (4 x contact + point), or -1
};
// A recorded run's branch decisions per step (the FP32 oracle's, which are the device's): with them
// the forward takes every clamp and threshold the recorded way, so its derivatives are those of
// the step over the frozen active set.
struct StepDecisions {
    std::vector<uint8_t> solve;      // [substep][iteration][contact][point]
    std::vector<uint8_t> position;   // [substep][iteration][contact][point]
    std::vector<uint8_t> integrate;  // [substep][row]
    std::vector<uint8_t> target;     // [contact][point]
};
// A recorded run's primal values (the FP32 oracle's, which are the device's): with them the forward
// evaluates its derivatives along that run instead of along its own FP64 values, so they are what
// the device's adjoint transposes. Per step: states at each substep's start [substep][row][13],
// velocities at each velocity iteration's start [substep][iteration][row][6], accumulated impulses
// there [substep][iteration][contact][point][3], resolutions at each position iteration's start
// [substep][iteration][row][3].
struct StepSnapshots {
    std::vector<float> state, vel, acc, res;
};
inline void snap(double& x, double v) { x = v; }
template <int K> void snap(Dual<K>& x, double v) { x.v = v; }

struct Problem {
    Params p;
    std::vector<BodyConst> bodies;
    std::vector<std::vector<ContactIn>> steps;
    std::vector<double> target;  // 3 per row: the loss's target final positions
    std::vector<StepDecisions> decisions;  // empty: every branch decided by the values
    std::vector<StepSnapshots> snapshots;  // empty: the forward's own values
    std::vector<float> final_state;        // with snapshots: the run's final states (13 per row)
};

template <class T>
struct State {
    std::vector<V3<T>> x, v, w;
    std::vector<Q4<T>> q;
};
template <class T>
struct Theta {
    std::vector<T> inverse_mass;       // per row
    std::vector<T> inverse_inertia;    // 6 per row
    std::vector<T> friction;           // per contact group
    State<T> start;
};

template <class T>
struct Arms {
    V3<T> ra[4], rb[4];
    T normal_mass[4], truth[4], t1_mass[4], t2_mass[4], twist_mass;
    V3<T> t1, t2;
};

template <class T>
void tangents(const V3<T>& n, V3<T>* t1, V3<T>* t2) {
    V3<T> t = std::fabs(val(n.x)) > 0.9 ? V3<T>{T(0.0), T(1.0), T(0.0)} : V3<T>{T(1.0), T(0.0), T(0.0)};
    V3<T> c = cross(n, t);
    *t1 = c / length(c);
    *t2 = cross(n, *t1);
}

// One body as a contact block sees it: inverse mass and world inverse inertia, zero when inert.
template <class T>
struct BlockBody {
    V3<T> x, v, w, com_world;
    Q4<T> q;
    T im;
    const T* ii;
    T split;  // contacts touching the body this step (mass splitting)
    bool inert;
    V3<T> iinv(const V3<T>& u, bool split_mass) const {
        if (inert) return zero3<T>();
        V3<T> local = quat_rotate(quat_conj(q), u);
        V3<T> r = quat_rotate(q, sym_apply(ii, local));
        return split_mass ? r * split : r;
    }
    T inverse_mass(bool split_mass) const { return inert ? T(0.0) : (split_mass ? im * split : im); }
};

template <class T>
T run(const Problem& P, const Theta<T>& th, State<T>* final_state) {
    const Params& p = P.p;
    const size_t n = P.bodies.size();
    State<T> s = th.start;
    const T dt = T(p.dt);
    const T h = T(p.dt / (double)p.substeps);
    std::vector<std::vector<V3<T>>> acc_prev;  // acc_out of the previous step, 4 per contact
    for (size_t step = 0; step < P.steps.size(); ++step) {
        const std::vector<ContactIn>& cs = P.steps[step];
        const size_t c = cs.size();
        const StepDecisions* dec = P.decisions.empty() ? nullptr : &P.decisions[step];
        const StepSnapshots* sn = P.snapshots.empty() ? nullptr : &P.snapshots[step];
        auto snap_states = [&](uint32_t sub) {
            if (!sn) return;
            for (size_t r = 0; r < n; ++r) {
                if (!P.bodies[r].dynamic) continue;
                const float* o = &sn->state[((size_t)sub * n + r) * 13];
                snap(s.x[r].x, o[0]); snap(s.x[r].y, o[1]); snap(s.x[r].z, o[2]);
                snap(s.q[r].x, o[3]); snap(s.q[r].y, o[4]); snap(s.q[r].z, o[5]); snap(s.q[r].w, o[6]);
                snap(s.v[r].x, o[7]); snap(s.v[r].y, o[8]); snap(s.v[r].z, o[9]);
                snap(s.w[r].x, o[10]); snap(s.w[r].y, o[11]); snap(s.w[r].z, o[12]);
            }
        };
        snap_states(0);
        // depths of the frozen contacts at this step's start, target speeds, block counts, acc_in
        std::vector<T> depth(4 * c, T(0.0)), target(4 * c, T(0.0));
        std::vector<V3<T>> acc(4 * c, zero3<T>());
        std::vector<uint32_t> counts(n, 0u);
        for (size_t i = 0; i < c; ++i) {
            const ContactIn& k = cs[i];
            if (!k.resolves) continue;
            counts[k.a] += 1u;
            counts[k.b] += 1u;
        }
        for (size_t i = 0; i < c; ++i) {
            const ContactIn& k = cs[i];
            const V3<T> nrm{T(k.normal[0]), T(k.normal[1]), T(k.normal[2])};
            for (uint32_t pi = 0; pi < k.count; ++pi) {
                const V3<T> la{T(k.la[pi][0]), T(k.la[pi][1]), T(k.la[pi][2])};
                const V3<T> lb{T(k.lb[pi][0]), T(k.lb[pi][1]), T(k.lb[pi][2])};
                V3<T> pa = s.x[k.a] + quat_rotate(s.q[k.a], la);
                V3<T> pb = s.x[k.b] + quat_rotate(s.q[k.b], lb);
                depth[4 * i + pi] = T(k.depth[pi]) + dot(nrm, pa - pb);
                int32_t src = k.source[pi];
                if (src >= 0 && step > 0) {
                    acc[4 * i + pi] = acc_prev[(size_t)src / 4][(size_t)src % 4];
                } else {
                    acc[4 * i + pi] = V3<T>{T(k.acc[pi][0]), T(k.acc[pi][1]), T(k.acc[pi][2])};
                }
            }
            if (!k.resolves) continue;
            // solver_blocks.wgsl:24-48 target speeds, from the velocities at the step's start
            for (uint32_t pi = 0; pi < k.count; ++pi) {
                const V3<T> pos{T(k.position[pi][0]), T(k.position[pi][1]), T(k.position[pi][2])};
                auto point_velocity = [&](uint32_t row) {
                    V3<T> com = s.x[row] + quat_rotate(s.q[row], V3<T>{T(P.bodies[row].com[0]), T(P.bodies[row].com[1]),
                                                                      T(P.bodies[row].com[2])});
                    return s.v[row] + cross(s.w[row], pos - com);
                };
                T speed = dot(point_velocity(k.b) - point_velocity(k.a), nrm);
                T d = depth[4 * i + pi];
                const bool from_depth = dec ? dec->target[4 * i + pi] == 1u : val(d) < 0.0;
                const bool from_restitution = dec ? dec->target[4 * i + pi] == 2u : val(speed) < -p.restitution_threshold;
                if (from_depth) {
                    target[4 * i + pi] = d / dt;
                } else if (from_restitution) {
                    target[4 * i + pi] = -speed * T(k.restitution);
                }
            }
        }
        auto block_body = [&](uint32_t row) {
            BlockBody<T> b;
            b.x = s.x[row];
            b.q = s.q[row];
            b.v = s.v[row];
            b.w = s.w[row];
            b.com_world = s.x[row] + quat_rotate(s.q[row], V3<T>{T(P.bodies[row].com[0]), T(P.bodies[row].com[1]),
                                                                T(P.bodies[row].com[2])});
            b.im = th.inverse_mass[row];
            b.ii = &th.inverse_inertia[6 * row];
            b.split = T((double)std::max(counts[row], 1u));
            b.inert = !P.bodies[row].dynamic;
            return b;
        };
        std::vector<V3<T>> resolution(n, zero3<T>());
        auto snap_iteration = [&](uint32_t sub, uint32_t it) {
            if (!sn) return;
            for (size_t r = 0; r < n; ++r) {
                if (!P.bodies[r].dynamic) continue;
                const float* o = &sn->vel[(((size_t)sub * p.iterations + it) * n + r) * 6];
                snap(s.v[r].x, o[0]); snap(s.v[r].y, o[1]); snap(s.v[r].z, o[2]);
                snap(s.w[r].x, o[3]); snap(s.w[r].y, o[4]); snap(s.w[r].z, o[5]);
            }
            for (size_t i = 0; i < c; ++i) {
                for (uint32_t pi = 0; pi < 4; ++pi) {
                    const float* o = &sn->acc[((((size_t)sub * p.iterations + it) * c + i) * 4 + pi) * 3];
                    snap(acc[4 * i + pi].x, o[0]);
                    snap(acc[4 * i + pi].y, o[1]);
                    snap(acc[4 * i + pi].z, o[2]);
                }
            }
        };
        if (sn && p.iterations > 0) {  // the warm start reads the impulses iteration 0 starts from
            for (size_t i = 0; i < c; ++i) {
                for (uint32_t pi = 0; pi < 4; ++pi) {
                    const float* o = &sn->acc[(i * 4 + pi) * 3];
                    snap(acc[4 * i + pi].x, o[0]);
                    snap(acc[4 * i + pi].y, o[1]);
                    snap(acc[4 * i + pi].z, o[2]);
                }
            }
        }
        for (uint32_t sub = 0; sub < p.substeps; ++sub) {
            if (sub > 0) snap_states(sub);
            // substep_integrate.wgsl:15-76 (no force fields, no applied forces)
            for (size_t r = 0; r < n; ++r) {
                const BodyConst& b = P.bodies[r];
                if (!b.dynamic) continue;
                V3<T> velocity = s.v[r] + V3<T>{T(p.gravity[0]), T(p.gravity[1]), T(p.gravity[2])} * (T(b.gravity_scale) * h);
                V3<T> spin = s.w[r];
                V3<T> gyro = spin;
                const double* I = b.inertia;
                bool isotropic = I[1] == 0.0 && I[2] == 0.0 && I[4] == 0.0 && I[0] == I[3] && I[3] == I[5];
                const T* ii = &th.inverse_inertia[6 * r];
                if (!isotropic) {
                    T It[6];
                    for (int k = 0; k < 6; ++k) It[k] = T(I[k]);
                    V3<T> body_spin = quat_rotate(quat_conj(s.q[r]), spin);
                    V3<T> momentum = sym_apply(It, body_spin);
                    V3<T> x = cross(body_spin, momentum);
                    if (!(val(x.x) == 0.0 && val(x.y) == 0.0 && val(x.z) == 0.0)) {
                        V3<T> solved = momentum;
                        for (int it = 0; it < 4; ++it) {
                            V3<T> mid = (momentum + solved) * T(0.5);
                            solved = rotate_about(-sym_apply(ii, mid) * h, momentum);
                        }
                        gyro = quat_rotate(s.q[r], sym_apply(ii, solved));
                    }
                }
                V3<T> angular = gyro;
                T speed = length(velocity);
                const uint8_t clamps = dec ? dec->integrate[(size_t)sub * n + r] : 0u;
                if (dec ? (clamps & 1u) != 0u : val(speed) > p.max_velocity) velocity = velocity * (T(p.max_velocity) / speed);
                T spin_speed = length(angular);
                if (dec ? (clamps & 2u) != 0u : val(spin_speed) > p.max_angular_velocity)
                    angular = angular * (T(p.max_angular_velocity) / spin_speed);
                s.v[r] = velocity / (T(1.0) + T(b.linear_damping) * h);
                s.w[r] = angular / (T(1.0) + T(b.angular_damping) * h);
            }
            // solver_contact_block.wgsl:24-80: arms and effective masses at this substep's poses
            std::vector<Arms<T>> arms(c);
            for (size_t i = 0; i < c; ++i) {
                const ContactIn& k = cs[i];
                if (!k.resolves) continue;
                BlockBody<T> f = block_body(k.a), g = block_body(k.b);
                Arms<T>& m = arms[i];
                const V3<T> nrm{T(k.normal[0]), T(k.normal[1]), T(k.normal[2])};
                tangents(nrm, &m.t1, &m.t2);
                V3<T> reach_f = zero3<T>(), reach_s = zero3<T>();
                for (uint32_t pi = 0; pi < k.count; ++pi) {
                    const V3<T> la{T(k.la[pi][0]), T(k.la[pi][1]), T(k.la[pi][2])};
                    const V3<T> lb{T(k.lb[pi][0]), T(k.lb[pi][1]), T(k.lb[pi][2])};
                    m.ra[pi] = (quat_rotate(f.q, la) + f.x) - f.com_world;
                    m.rb[pi] = (quat_rotate(g.q, lb) + g.x) - g.com_world;
                    reach_f = reach_f + m.ra[pi];
                    reach_s = reach_s + m.rb[pi];
                }
                T count = T((double)std::max(k.count, 1u));
                V3<T> spread_f = f.iinv(cross(reach_f, nrm), true), spread_s = g.iinv(cross(reach_s, nrm), true);
                auto momentum_mass = [&](const V3<T>& ra, const V3<T>& rb, const V3<T>& axis, bool split) {
                    V3<T> rax = cross(ra, axis), rbx = cross(rb, axis);
                    return f.inverse_mass(split) + g.inverse_mass(split) + dot(rax, f.iinv(rax, split)) + dot(rbx, g.iinv(rbx, split));
                };
                for (uint32_t pi = 0; pi < k.count; ++pi) {
                    m.normal_mass[pi] = count * (f.inverse_mass(true) + g.inverse_mass(true)) + dot(spread_f, cross(m.ra[pi], nrm))
                        + dot(spread_s, cross(m.rb[pi], nrm));
                    m.truth[pi] = momentum_mass(m.ra[pi], m.rb[pi], nrm, false);
                    m.t1_mass[pi] = momentum_mass(m.ra[pi], m.rb[pi], m.t1, true) * count;
                    m.t2_mass[pi] = momentum_mass(m.ra[pi], m.rb[pi], m.t2, true) * count;
                }
                m.twist_mass = dot(nrm, f.iinv(nrm, true)) + dot(nrm, g.iinv(nrm, true));
            }
            auto apply_deltas = [&](const std::vector<V3<T>>& dv, const std::vector<V3<T>>& dw) {
                for (size_t r = 0; r < n; ++r) {
                    if (!P.bodies[r].dynamic) continue;
                    s.v[r] = s.v[r] + dv[r];
                    s.w[r] = s.w[r] + dw[r];
                }
            };
            if (sub == 0) {
                // solver_contact_block.wgsl:195-233 warm start
                std::vector<V3<T>> dv(n, zero3<T>()), dw(n, zero3<T>());
                for (size_t i = 0; i < c; ++i) {
                    const ContactIn& k = cs[i];
                    if (!k.resolves) continue;
                    BlockBody<T> f = block_body(k.a), g = block_body(k.b);
                    if (f.inert && g.inert) continue;
                    const V3<T> nrm{T(k.normal[0]), T(k.normal[1]), T(k.normal[2])};
                    const Arms<T>& m = arms[i];
                    for (uint32_t pi = 0; pi < k.count; ++pi) {
                        const V3<T>& a = acc[4 * i + pi];
                        V3<T> j = nrm * a.x + m.t1 * a.y + m.t2 * a.z;
                        if (!f.inert) {
                            dv[k.a] = dv[k.a] - j * f.im;
                            dw[k.a] = dw[k.a] - f.iinv(cross(m.ra[pi], j), false);
                        }
                        if (!g.inert) {
                            dv[k.b] = dv[k.b] + j * g.im;
                            dw[k.b] = dw[k.b] + g.iinv(cross(m.rb[pi], j), false);
                        }
                    }
                }
                apply_deltas(dv, dw);
            }
            for (uint32_t it = 0; it < p.iterations; ++it) {
                snap_iteration(sub, it);
                // solver_contact_block.wgsl:6-193, Jacobi over the blocks, then solver_block_apply.wgsl
                std::vector<V3<T>> dv(n, zero3<T>()), dw(n, zero3<T>());
                std::vector<V3<T>> next(acc);
                for (size_t i = 0; i < c; ++i) {
                    const ContactIn& k = cs[i];
                    if (!k.resolves) continue;
                    BlockBody<T> f = block_body(k.a), g = block_body(k.b);
                    if (f.inert && g.inert) continue;
                    const V3<T> nrm{T(k.normal[0]), T(k.normal[1]), T(k.normal[2])};
                    const Arms<T>& m = arms[i];
                    const T mu = th.friction[k.group];
                    V3<T> fv = zero3<T>(), fw = zero3<T>(), sv = zero3<T>(), sw = zero3<T>();  // the block's changes
                    T normal_total = T(0.0);
                    for (uint32_t pi = 0; pi < k.count; ++pi) normal_total = normal_total + wmax(acc[4 * i + pi].x, T(0.0));
                    for (uint32_t pi = 0; pi < k.count; ++pi) {
                        const V3<T>& a = acc[4 * i + pi];
                        V3<T> rel = (g.v + cross(g.w, m.rb[pi])) - (f.v + cross(f.w, m.ra[pi]));
                        T ns = dot(rel, nrm);
                        T goal = target[4 * i + pi];
                        T delta;
                        if (k.relaxation <= 0.0) {
                            delta = (goal - ns) / m.normal_mass[pi];
                        } else {
                            // core.wgsl:326-345 (soft contact)
                            T bias = wmax(depth[4 * i + pi] / dt, goal);
                            T drag = T(2.0 * k.damping_ratio * k.relaxation) / dt;
                            T softness = T(k.relaxation * k.relaxation) * m.truth[pi] / (dt * dt);
                            T prior = ns - a.x * m.truth[pi];
                            T wanted = (bias - (T(1.0) + drag) * prior) / (softness + (T(1.0) + drag) * m.truth[pi]);
                            delta = m.truth[pi] * (wanted - a.x) / m.normal_mass[pi];
                        }
                        T an, at1, at2, rem;
                        T limit, u1, u2;
                        if (dec) {
                            const uint8_t f = dec->solve[(((size_t)sub * p.iterations + it) * c + i) * 4 + pi];
                            an = (f & 1u) ? a.x + delta : T(0.0);
                            limit = mu * an;
                            u1 = a.y - dot(rel, m.t1) / m.t1_mass[pi];
                            at1 = (f & 2u) ? limit : ((f & 4u) ? -limit : u1);
                            rem = (f & 8u) ? sqrt(wmax(limit * limit - at1 * at1, T(0.0))) : T(0.0);
                            u2 = a.z - dot(rel, m.t2) / m.t2_mass[pi];
                            at2 = (f & 16u) ? rem : ((f & 32u) ? -rem : u2);
                        } else {
                            an = wmax(T(0.0), a.x + delta);
                            limit = mu * an;
                            u1 = a.y - dot(rel, m.t1) / m.t1_mass[pi];
                            at1 = wclamp(u1, -limit, limit);
                            rem = sqrt(wmax(limit * limit - at1 * at1, T(0.0)));
                            u2 = a.z - dot(rel, m.t2) / m.t2_mass[pi];
                            at2 = wclamp(u2, -rem, rem);
                        }
                        V3<T> j = nrm * (an - a.x) + m.t1 * (at1 - a.y) + m.t2 * (at2 - a.z);
                        next[4 * i + pi] = V3<T>{an, at1, at2};
                        fv = fv - j * f.inverse_mass(false);
                        fw = fw - f.iinv(cross(m.ra[pi], j), false);
                        sv = sv + j * g.inverse_mass(false);
                        sw = sw + g.iinv(cross(m.rb[pi], j), false);
                    }
                    // rolling and twist friction over the block's updated spins
                    V3<T> rel_spin = (g.w + sw) - (f.w + fw);
                    V3<T> planar = rel_spin - nrm * dot(rel_spin, nrm);
                    T planar_len = length(planar);
                    if (val(planar_len) > 1e-6) {
                        V3<T> axis = planar / planar_len;
                        T mass = dot(axis, f.iinv(axis, true)) + dot(axis, g.iinv(axis, true));
                        if (val(mass) > 0.0) {
                            T limit = T(k.rolling) * normal_total;
                            T applied = wclamp(-planar_len / mass, -limit, limit);
                            fw = fw - f.iinv(axis * applied, false);
                            sw = sw + g.iinv(axis * applied, false);
                        }
                    }
                    T twist = dot(rel_spin, nrm);
                    if (std::fabs(val(twist)) > 1e-6 && val(m.twist_mass) > 0.0) {
                        T limit = T(k.spin) * normal_total;
                        T applied = wclamp(-twist / m.twist_mass, -limit, limit);
                        fw = fw - f.iinv(nrm * applied, false);
                        sw = sw + g.iinv(nrm * applied, false);
                    }
                    if (!f.inert) {
                        dv[k.a] = dv[k.a] + fv;
                        dw[k.a] = dw[k.a] + fw;
                    }
                    if (!g.inert) {
                        dv[k.b] = dv[k.b] + sv;
                        dw[k.b] = dw[k.b] + sw;
                    }
                }
                acc.swap(next);
                apply_deltas(dv, dw);
            }
            // substep_advance.wgsl:6-13
            for (size_t r = 0; r < n; ++r) {
                if (!P.bodies[r].dynamic) continue;
                s.x[r] = s.x[r] + s.v[r] * h;
                Q4<T> spin{s.w[r].x, s.w[r].y, s.w[r].z, T(0.0)};
                Q4<T> d = quat_mul(spin, s.q[r]);
                T half = T(0.5) * h;
                s.q[r] = normalize4(Q4<T>{s.q[r].x + half * d.x, s.q[r].y + half * d.y, s.q[r].z + half * d.z, s.q[r].w + half * d.w});
            }
            // position_correction.wgsl:5-46 + position_block.wgsl:11-33, position_apply.wgsl:12-27
            for (uint32_t it = 0; it < p.position_iterations; ++it) {
                if (sn) {
                    for (size_t r = 0; r < n; ++r) {
                        const float* o = &sn->res[(((size_t)sub * p.position_iterations + it) * n + r) * 3];
                        snap(resolution[r].x, o[0]);
                        snap(resolution[r].y, o[1]);
                        snap(resolution[r].z, o[2]);
                    }
                }
                std::vector<V3<T>> sum(n, zero3<T>());
                std::vector<uint32_t> contributions(n, 0u);
                for (size_t i = 0; i < c; ++i) {
                    const ContactIn& k = cs[i];
                    if (!k.resolves || k.relaxation > 0.0) continue;
                    const bool fa = P.bodies[k.a].dynamic, fb = P.bodies[k.b].dynamic;
                    T ima = fa ? th.inverse_mass[k.a] : T(0.0);
                    T imb = fb ? th.inverse_mass[k.b] : T(0.0);
                    const V3<T> nrm{T(k.normal[0]), T(k.normal[1]), T(k.normal[2])};
                    T resolved = dot(nrm, resolution[k.b] - resolution[k.a]);
                    V3<T> total = zero3<T>();
                    uint32_t contributing = 0;
                    for (uint32_t pi = 0; pi < k.count; ++pi) {
                        T error = depth[4 * i + pi] - T(p.slop) - resolved;
                        T kk = ima + imb;
                        if (dec) {
                            if (dec->position[(((size_t)sub * p.position_iterations + it) * c + i) * 4 + pi] == 0u) continue;
                        } else {
                            error = wmax(error, T(0.0));
                            if (!(val(error) > 0.0)) continue;
                            if (val(kk) == 0.0) continue;
                        }
                        total = total + nrm * (T(p.relaxation) * error / kk);
                        contributing += 1;
                    }
                    if (contributing == 0u) continue;
                    V3<T> correction = total / T((double)contributing);
                    V3<T> lf = -correction * ima, ls = correction * imb;
                    if (!dec && !(val(dot(lf, lf)) > 0.0 || val(dot(ls, ls)) > 0.0)) continue;
                    contributions[k.a] += 1u;
                    contributions[k.b] += 1u;
                    sum[k.a] = sum[k.a] + lf;
                    sum[k.b] = sum[k.b] + ls;
                }
                for (size_t r = 0; r < n; ++r) {
                    if (contributions[r] == 0u || !P.bodies[r].dynamic) continue;
                    V3<T> applied = sum[r] / T((double)contributions[r]);
                    s.x[r] = s.x[r] + applied;
                    s.q[r] = normalize4(s.q[r]);
                    resolution[r] = resolution[r] + applied;
                }
            }
        }
        acc_prev.assign(c, std::vector<V3<T>>(4, zero3<T>()));
        for (size_t i = 0; i < c; ++i) {
            for (uint32_t pi = 0; pi < 4; ++pi) acc_prev[i][pi] = acc[4 * i + pi];
        }
    }
    if (!P.final_state.empty()) {
        for (size_t r = 0; r < n; ++r) {
            if (!P.bodies[r].dynamic) continue;
            const float* o = &P.final_state[r * 13];
            snap(s.x[r].x, o[0]); snap(s.x[r].y, o[1]); snap(s.x[r].z, o[2]);
        }
    }
    T loss = T(0.0);
    for (size_t r = 0; r < n; ++r) {
        if (!P.bodies[r].dynamic) continue;
        V3<T> d = s.x[r] - V3<T>{T(P.target[3 * r]), T(P.target[3 * r + 1]), T(P.target[3 * r + 2])};
        loss = loss + dot(d, d);
    }
    if (final_state) *final_state = s;
    return loss;
}

// ---- flat inputs from Python ----
// bodies: 20 doubles per row: inverse_mass, inverse_inertia[6], com[3], gravity_scale, linear_damping,
//   angular_damping, inertia[6], dynamic (0/1)
// state: 13 doubles per row: position[3], orientation[4] (x, y, z, w), velocity[3], angular_velocity[3]
// params: dt, gravity[3], slop, relaxation, restitution_threshold, max_velocity, max_angular_velocity,
//   substeps, iterations, position_iterations
// contacts (all steps back to back, counts[step] each): ints 5 per contact (a, b, count, group,
//   resolves), doubles 8 per contact (normal[3], restitution, rolling, spin, relaxation, damping_ratio)
//   and 16 per point x 4 (la[3], lb[3], depth, position[3], acc[3], pad[3]), sources 4 per contact
//   (index into the previous step's points, -1 = not relayed)
Problem make_problem(uint32_t n, const double* bodies, const double* params, uint32_t steps, const uint32_t* counts,
                     const int32_t* cint, const double* cdouble, const double* cpoints, const int32_t* sources,
                     const double* target, const uint8_t* decisions, const float* snapshots, const float* final_state) {
    Problem P;
    P.p.dt = params[0];
    for (int k = 0; k < 3; ++k) P.p.gravity[k] = params[1 + k];
    P.p.slop = params[4];
    P.p.relaxation = params[5];
    P.p.restitution_threshold = params[6];
    P.p.max_velocity = params[7];
    P.p.max_angular_velocity = params[8];
    P.p.substeps = (uint32_t)params[9];
    P.p.iterations = (uint32_t)params[10];
    P.p.position_iterations = (uint32_t)params[11];
    P.bodies.resize(n);
    for (uint32_t r = 0; r < n; ++r) {
        const double* b = bodies + 20 * (size_t)r;
        BodyConst& c = P.bodies[r];
        for (int k = 0; k < 3; ++k) c.com[k] = b[7 + k];
        c.gravity_scale = b[10];
        c.linear_damping = b[11];
        c.angular_damping = b[12];
        for (int k = 0; k < 6; ++k) c.inertia[k] = b[13 + k];
        c.dynamic = b[19] != 0.0;
    }
    size_t base = 0;
    P.steps.resize(steps);
    for (uint32_t st = 0; st < steps; ++st) {
        P.steps[st].resize(counts[st]);
        for (uint32_t i = 0; i < counts[st]; ++i, ++base) {
            ContactIn& c = P.steps[st][i];
            const int32_t* ci = cint + 5 * base;
            const double* cd = cdouble + 8 * base;
            c.a = (uint32_t)ci[0];
            c.b = (uint32_t)ci[1];
            c.count = (uint32_t)ci[2];
            c.group = (uint32_t)ci[3];
            c.resolves = ci[4] != 0;
            for (int k = 0; k < 3; ++k) c.normal[k] = cd[k];
            c.restitution = cd[3];
            c.rolling = cd[4];
            c.spin = cd[5];
            c.relaxation = cd[6];
            c.damping_ratio = cd[7];
            for (int pi = 0; pi < 4; ++pi) {
                const double* pt = cpoints + 64 * base + 16 * pi;
                for (int k = 0; k < 3; ++k) {
                    c.la[pi][k] = pt[k];
                    c.lb[pi][k] = pt[3 + k];
                    c.position[pi][k] = pt[7 + k];
                    c.acc[pi][k] = pt[10 + k];
                }
                c.depth[pi] = pt[6];
                c.source[pi] = sources[4 * base + pi];
            }
        }
    }
    P.target.assign(target, target + 3 * (size_t)n);
    if (decisions) {
        // per step, back to back: solve, position, integrate, target flags
        const size_t K = P.p.substeps, I = P.p.iterations, PI = P.p.position_iterations;
        P.decisions.resize(steps);
        const uint8_t* at = decisions;
        for (uint32_t st = 0; st < steps; ++st) {
            const size_t c = counts[st];
            StepDecisions& d = P.decisions[st];
            d.solve.assign(at, at + K * I * 4 * c);
            at += K * I * 4 * c;
            d.position.assign(at, at + K * PI * 4 * c);
            at += K * PI * 4 * c;
            d.integrate.assign(at, at + K * n);
            at += K * n;
            d.target.assign(at, at + 4 * c);
            at += 4 * c;
        }
    }
    if (snapshots) {
        // per step, back to back: states, velocities, impulses, resolutions
        const size_t K = P.p.substeps, I = P.p.iterations, PI = P.p.position_iterations;
        P.snapshots.resize(steps);
        const float* at = snapshots;
        for (uint32_t st = 0; st < steps; ++st) {
            const size_t c = counts[st];
            StepSnapshots& sn = P.snapshots[st];
            sn.state.assign(at, at + K * n * 13);
            at += K * n * 13;
            sn.vel.assign(at, at + K * I * n * 6);
            at += K * I * n * 6;
            sn.acc.assign(at, at + K * I * c * 12);
            at += K * I * c * 12;
            sn.res.assign(at, at + K * PI * n * 3);
            at += K * PI * n * 3;
        }
    }
    if (final_state) P.final_state.assign(final_state, final_state + 13 * (size_t)n);
    return P;
}

template <class T>
Theta<T> make_theta(const Problem& P, const double* bodies, const double* friction, uint32_t groups, const double* state) {
    const size_t n = P.bodies.size();
    Theta<T> th;
    th.inverse_mass.resize(n);
    th.inverse_inertia.resize(6 * n);
    for (size_t r = 0; r < n; ++r) {
        th.inverse_mass[r] = T(bodies[20 * r]);
        for (int k = 0; k < 6; ++k) th.inverse_inertia[6 * r + k] = T(bodies[20 * r + 1 + k]);
    }
    th.friction.resize(groups);
    for (uint32_t g = 0; g < groups; ++g) th.friction[g] = T(friction[g]);
    th.start.x.resize(n);
    th.start.q.resize(n);
    th.start.v.resize(n);
    th.start.w.resize(n);
    for (size_t r = 0; r < n; ++r) {
        const double* s = state + 13 * r;
        th.start.x[r] = V3<T>{T(s[0]), T(s[1]), T(s[2])};
        th.start.q[r] = Q4<T>{T(s[3]), T(s[4]), T(s[5]), T(s[6])};
        th.start.v[r] = V3<T>{T(s[7]), T(s[8]), T(s[9])};
        th.start.w[r] = V3<T>{T(s[10]), T(s[11]), T(s[12])};
    }
    return th;
}

constexpr int kLanes = 8;

}  // namespace adj

extern "C" {

// The FP64 forward over the frozen contact sets: returns the loss and writes the final state
// (13 doubles per row) when out_state is not null. friction: one value per contact group.
// decisions: null (branches decided by the values) or a recorded run's flags per step; snapshots and
// final_state: null, or a recorded run's primal values along which the derivatives are taken.
double adj_forward(uint32_t n, const double* bodies, const double* params, uint32_t steps, const uint32_t* counts,
                   const int32_t* cint, const double* cdouble, const double* cpoints, const int32_t* sources,
                   const double* target, const uint8_t* decisions, const float* snapshots, const float* final_state,
                   const double* friction, uint32_t groups, const double* state, double* out_state) {
    adj::Problem P = adj::make_problem(n, bodies, params, steps, counts, cint, cdouble, cpoints, sources, target, decisions,
                                       snapshots, final_state);
    adj::Theta<double> th = adj::make_theta<double>(P, bodies, friction, groups, state);
    adj::State<double> fin;
    double loss = adj::run(P, th, &fin);
    if (out_state) {
        for (uint32_t r = 0; r < n; ++r) {
            double* o = out_state + 13 * (size_t)r;
            o[0] = fin.x[r].x; o[1] = fin.x[r].y; o[2] = fin.x[r].z;
            o[3] = fin.q[r].x; o[4] = fin.q[r].y; o[5] = fin.q[r].z; o[6] = fin.q[r].w;
            o[7] = fin.v[r].x; o[8] = fin.v[r].y; o[9] = fin.v[r].z;
            o[10] = fin.w[r].x; o[11] = fin.w[r].y; o[12] = fin.w[r].z;
        }
    }
    return loss;
}

// Directional derivatives of the loss (forward mode, FP64) along `directions` tangent vectors of
// the parameter vector [inverse_mass (n), inverse_inertia (6n), friction (groups), state (13n)],
// directions x (20n + groups) doubles; writes one derivative per direction into out.
void adj_directional(uint32_t n, const double* bodies, const double* params, uint32_t steps, const uint32_t* counts,
                     const int32_t* cint, const double* cdouble, const double* cpoints, const int32_t* sources,
                     const double* target, const uint8_t* decisions, const float* snapshots, const float* final_state,
                     const double* friction, uint32_t groups, const double* state, uint32_t directions,
                     const double* tangent, double* out) {
    using D = adj::Dual<adj::kLanes>;
    adj::Problem P = adj::make_problem(n, bodies, params, steps, counts, cint, cdouble, cpoints, sources, target, decisions,
                                       snapshots, final_state);
    const size_t dim = 20 * (size_t)n + groups;
    for (uint32_t first = 0; first < directions; first += adj::kLanes) {
        adj::Theta<D> th = adj::make_theta<D>(P, bodies, friction, groups, state);
        const uint32_t lanes = std::min<uint32_t>(adj::kLanes, directions - first);
        for (uint32_t l = 0; l < lanes; ++l) {
            const double* t = tangent + (size_t)(first + l) * dim;
            for (uint32_t r = 0; r < n; ++r) {
                th.inverse_mass[r].d[l] = t[r];
                for (int k = 0; k < 6; ++k) th.inverse_inertia[6 * r + k].d[l] = t[n + 6 * (size_t)r + k];
            }
            for (uint32_t g = 0; g < groups; ++g) th.friction[g].d[l] = t[7 * (size_t)n + g];
            const double* ts = t + 7 * (size_t)n + groups;
            for (uint32_t r = 0; r < n; ++r) {
                const double* v = ts + 13 * (size_t)r;
                th.start.x[r].x.d[l] = v[0]; th.start.x[r].y.d[l] = v[1]; th.start.x[r].z.d[l] = v[2];
                th.start.q[r].x.d[l] = v[3]; th.start.q[r].y.d[l] = v[4]; th.start.q[r].z.d[l] = v[5]; th.start.q[r].w.d[l] = v[6];
                th.start.v[r].x.d[l] = v[7]; th.start.v[r].y.d[l] = v[8]; th.start.v[r].z.d[l] = v[9];
                th.start.w[r].x.d[l] = v[10]; th.start.w[r].y.d[l] = v[11]; th.start.w[r].z.d[l] = v[12];
            }
        }
        D loss = adj::run<D>(P, th, nullptr);
        for (uint32_t l = 0; l < lanes; ++l) out[first + l] = loss.d[l];
    }
}

}  // extern "C"
