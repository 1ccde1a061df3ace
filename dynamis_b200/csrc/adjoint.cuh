// adjoint.cuh - the adjoint of the rigid-body step over its frozen active contact set (sm_100a).
//
// Differentiates one World::step from the state its substeps start from to the state it ends in:
// substep integration (substep_integrate.wgsl:15-76), the warm start and Jacobi contact blocks
// (solver_contact_block.wgsl:6-233 with core.wgsl:326-345, hard contacts), advance
// (substep_advance.wgsl:6-13) and position correction (position_correction.wgsl:5-46,
// position_block.wgsl:11-33, position_apply.wgsl:12-27), plus the target speeds of
// solver_blocks.wgsl:24-48 and the relay of accumulated impulses from the previous step
// (contact_relay.wgsl:34-72). The contact set a step's narrowphase produced is frozen: which pairs
// touch, their normals, their points' anchors in each body's frame, which clamp of the solve was
// active. A point's depth moves with the bodies to first order, d = d0 + n . (p_a - p_b), p_a and
// p_b being the point's anchors carried by each body (both at the contact point when the
// narrowphase ran). The fixed-point delta accumulation (core.wgsl:6-12) is differentiated as the
// exact sum it stands for.
//
// Forward, a taped step (record_step with a tape) snapshots what the reverse needs into one slot of
// the tape: the contact set with its target speeds and relay sources, the body rows at each
// substep's start and at the step's end, the velocities and accumulated impulses at each velocity
// iteration's start, and the resolution and contribution counts of each position iteration. The
// iteration snapshots are written by the forward kernels themselves (k_solve, k_position_fused,
// k_papply_last through DeviceWorld::tape), and only for the rows and contacts a contact block
// solves: the reverse reads no other entry of them.
// Backward, one captured graph reverses one step: it takes the slot below the tape's counter and
// runs the reverse of every pass in reverse order, one thread per contact block or body row, the
// same decomposition as the forward; contact threads add their contributions to shared rows with
// float atomics into separate buffers that row kernels fold in.
//
// Where the clamp of the friction cone is not differentiable, the adjoint takes a subgradient: at
// the branch point of the tangent-2 limit (kTangentLimitFloor) that limit is locally constant.
//
// Supported: hard contacts without rolling or spin friction, bodies with isotropic inverse inertia
// (the world inverse inertia then does not depend on the orientation), no joints, sleeping off.
// A contact outside that set raises DYN_STATUS_ADJOINT_UNSUPPORTED and is skipped.
#pragma once

#include "step.cuh"

namespace dyn {

constexpr uint32_t kNoRelay = 0xFFFFFFFFu;
// Below this fraction of the friction limit the tangent-2 limit sqrt(limit^2 - tangent_1^2) passes
// no derivative: at its branch point (tangent 1 at the limit) d/d limit = limit / sqrt(...) is
// unbounded, and one rounding of limit^2 - tangent_1^2 changes it by its own size. There the
// adjoint takes the subgradient of a locally constant tangent-2 limit.
constexpr float kTangentLimitFloor = 0.05f;

// One segment of taped steps. Per step slot s: contacts [s][c], points [s][4c] (point p of contact i
// at p * c + i, the device layout), body rows [s][substeps + 1][n], velocity-iteration snapshots
// [s][substeps * iterations][...], position-iteration snapshots [s][substeps * piterations][n].
struct TapeView {
    uint32_t* slot;  // device counter: the slot a taped step writes, then the slot count
    uint32_t steps, substeps, iterations, piterations;
    size_t n, c;
    uint32_t* counts;  // [steps] contacts of the step
    uint4* rows;
    float4* normal;
    float4* mat;
    uint4* ids;
    float4* extra;
    float4* la;        // local anchor on the first body, narrowphase depth
    float4* lb;        // local anchor on the second body, target speed
    float4* pos;       // contact point (world), as the narrowphase placed it
    uint32_t* relay;   // source point (p * c + h) in the previous step of every point, or kNoRelay
    float4* acc;       // [s][substeps * iterations][4c] accumulated impulses at a velocity iteration's start
    BodyHot* hot;      // [s][substeps + 1][n]
    float4* vel;       // [s][substeps * iterations][2n] velocities, then angular velocities
    float4* res;       // [s][substeps * piterations][n] resolution at a position iteration's start
    uint32_t* cnt;     // [s][substeps * piterations][n] contributions counted by that iteration
    __device__ __forceinline__ size_t cs(uint32_t s) const { return (size_t)s * c; }
    __device__ __forceinline__ size_t ps(uint32_t s) const { return (size_t)s * 4 * c; }
    __device__ __forceinline__ const BodyHot* hot_at(uint32_t s, uint32_t k) const {
        return hot + ((size_t)s * (substeps + 1) + k) * n;
    }
    __device__ __forceinline__ const float4* vel_at(uint32_t s, uint32_t k, uint32_t it) const {
        return vel + ((size_t)s * substeps * iterations + (size_t)k * iterations + it) * 2 * n;
    }
    __device__ __forceinline__ const float4* acc_at(uint32_t s, uint32_t k, uint32_t it) const {
        return acc + ((size_t)s * substeps * iterations + (size_t)k * iterations + it) * 4 * c;
    }
    __device__ __forceinline__ size_t pslot(uint32_t s, uint32_t k, uint32_t it) const {
        return ((size_t)s * substeps * piterations + (size_t)k * piterations + it) * n;
    }
};

// Gradient buffers of a backward pass.
struct AdjView {
    float4* gx;  // [n] d loss / d position (xyz)
    float4* gq;  // [n] d loss / d orientation (xyzw)
    float4* gv;  // [n] d loss / d velocity
    float4* gw;  // [n] d loss / d angular velocity
    float4* gv_acc;  // [n] a velocity iteration's contributions to gv, gw (folded in by k_adj_vmerge)
    float4* gw_acc;
    float4* gres;      // [n] d loss / d resolution
    float4* gres_acc;  // [n] a position iteration's contributions to gres
    float4* gsum;      // [n] d loss / d (a position iteration's summed delta of the row)
    float* g_im;       // [n] d loss / d inverse mass (accumulated over the steps reversed)
    float* g_scale;    // [n] d loss / d scale of the inverse inertia tensor (d/dl L(l I^-1) at l = 1)
    float* g_friction; // [k] d loss / d collider friction
    float4* gacc[2];   // [4c] d loss / d accumulated impulses (normal, tangent 1, tangent 2): this step, previous
    uint32_t* acc_flip;  // device word: which gacc is this step's
    float4* g_ra;      // [4c] d loss / d arm on the first body (xyz), d loss / d normal mass (w), one substep
    float4* g_rb;      // [4c] d loss / d arm on the second body (xyz), d loss / d target speed (w, whole step)
    float2* g_m;       // [4c] d loss / d tangent-1 mass, tangent-2 mass
    float4* g_pt;      // [4c] d loss / d depth (y), whole step
    float4* g_param;   // [c] d loss / d inverse mass of the first and second body, of their inertia scales
    float4* t_arm_a;   // [4c] a substep's pose-only terms (k_adj_terms): arm on the first body, normal mass
    float4* t_arm_b;   // [4c] arm on the second body
    float4* t_mass;    // [4c] tangent-1 mass, tangent-2 mass, target speed
    float4* t_tan1;    // [c] tangent 1
    float4* t_tan2;    // [c] tangent 2, the block's kBlock* flags (w, as bits)
    float4* t_body;    // [c] inverse mass of the first and second body, their inverse inertia scalars (0 when inert)
    float* g_mu;       // [c] d loss / d contact friction
    uint32_t* status;
};

// ---- helpers ----
// d/dq of quat_rotate(q, v) (core.wgsl's form, 2(u.v)u + (s^2 - u.u)v + 2s(u x v)) against an output gradient g
__device__ __forceinline__ float4 quat_rotate_qgrad(float4 q, f3 v, f3 g) {
    const f3 u = xyz(q);
    const float s = q.w;
    const f3 gu = 2.0f * (dot(g, u) * v + dot(u, v) * g) - 2.0f * dot(g, v) * u + 2.0f * s * cross(v, g);
    const float gs = 2.0f * s * dot(g, v) + 2.0f * dot(g, cross(u, v));
    return mk4(gu, gs);
}
__device__ __forceinline__ void atomic_add3(float4* p, f3 v) {
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
    atomicAdd(&p->z, v.z);
}
__device__ __forceinline__ void atomic_add4(float4* p, float4 v) {
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
    atomicAdd(&p->z, v.z);
    atomicAdd(&p->w, v.w);
}
__device__ __forceinline__ f3 add3(float4 a, f3 b) { return xyz(a) + b; }
__device__ __forceinline__ bool row_live(const BodyHot& h) { return simulates(h.pos.w, h.aux.y) && h.aux.x == 0u; }
// A body row as the contact blocks of a substep saw it: its pose at the substep's start, velocities given.
__device__ __forceinline__ DBody tape_body(const BodyHot& h, float4 v, float4 w) {
    DBody b;
    b.position = xyz(h.pos);
    b.inverse_mass = h.pos.w;
    b.orientation = h.rot;
    b.velocity = xyz(v);
    b.angular_velocity = xyz(w);
    b.com = xyz(h.com);
    b.ii0 = h.ii0;
    b.ii1 = make_float2(h.ii1.x, h.ii1.y);
    b.sleeping = h.aux.x;
    b.flags = h.aux.y;
    return b;
}
// The block's bodies (block_bodies of step.cuh, from taped rows) and the pose-only terms
// k_solve_prepare computed for them, recomputed with the same expressions.
struct TapeBlock {
    DBody pf, ps, sf, ss;
    bool inert_f, inert_s;
    f3 normal, t1, t2;
    float friction;
    uint32_t count;
    f3 ra[4], rb[4];
    float nm[4], m1[4], m2[4];
    f3 reach_f, reach_s, spread_f, spread_s;
    float count_f;
};
// The block's bodies alone (what the impulses act on); tape_block adds the pose-only terms.
__device__ __forceinline__ void tape_block_bodies(const TapeView& t, uint32_t s, uint32_t k, uint32_t i, uint4 r,
                                                  const float4* vel, TapeBlock* b) {
    const BodyHot* hot = t.hot_at(s, k);
    const BodyHot& ha = hot[r.x];
    const BodyHot& hb = hot[r.y];
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    b->pf = tape_body(ha, vel ? vel[r.x] : zero, vel ? vel[t.n + r.x] : zero);
    b->ps = tape_body(hb, vel ? vel[r.y] : zero, vel ? vel[t.n + r.y] : zero);
    b->sf = split_body(b->pf, (float)max(ha.aux.z, 1u));
    b->ss = split_body(b->ps, (float)max(hb.aux.z, 1u));
    b->inert_f = dbody_inert(b->pf);
    b->inert_s = dbody_inert(b->ps);
    if (b->inert_f) {
        b->pf = dbody_frozen(b->pf);
        b->sf = dbody_frozen(b->sf);
    }
    if (b->inert_s) {
        b->ps = dbody_frozen(b->ps);
        b->ss = dbody_frozen(b->ss);
    }
    const float4 nf = t.normal[t.cs(s) + i];
    b->normal = xyz(nf);
    b->friction = nf.w;
    b->count = r.z & 0xFFu;
}
__device__ __forceinline__ void tape_block(const TapeView& t, uint32_t s, uint32_t k, uint32_t i, uint4 r, const float4* vel,
                                           TapeBlock* b) {
    tape_block_bodies(t, s, k, i, r, vel, b);
    make_tangents(b->normal, &b->t1, &b->t2);
    b->reach_f = s3(0.0f);
    b->reach_s = s3(0.0f);
    #pragma unroll
    for (uint32_t p = 0; p < 4u; ++p) if (p < b->count) {
        const size_t o = t.ps(s) + (size_t)p * t.c + i;
        b->ra[p] = arm(b->pf, xyz(t.la[o])) - dbody_com(b->pf);
        b->rb[p] = arm(b->ps, xyz(t.lb[o])) - dbody_com(b->ps);
        b->reach_f = b->reach_f + b->ra[p];
        b->reach_s = b->reach_s + b->rb[p];
    }
    b->count_f = (float)max(b->count, 1u);
    b->spread_f = dbody_iinv(b->sf, cross(b->reach_f, b->normal));
    b->spread_s = dbody_iinv(b->ss, cross(b->reach_s, b->normal));
    #pragma unroll
    for (uint32_t p = 0; p < 4u; ++p) if (p < b->count) {
        const f3 arm_f = cross(b->ra[p], b->normal);
        const f3 arm_s = cross(b->rb[p], b->normal);
        b->nm[p] = b->count_f * (b->sf.inverse_mass + b->ss.inverse_mass) + dot(b->spread_f, arm_f) + dot(b->spread_s, arm_s);
        b->m1[p] = momentum_mass_arms(b->sf, b->ss, b->ra[p], b->rb[p], b->t1) * b->count_f;
        b->m2[p] = momentum_mass_arms(b->sf, b->ss, b->ra[p], b->rb[p], b->t2) * b->count_f;
    }
}
// What k_adj_terms found of a contact block for one substep (AdjView::t_tan2.w): the velocity
// iterations reverse it (resolves, supported, not both bodies inert), which body is inert, and
// whether the position passes correct it (resolves, hard contact).
constexpr uint32_t kBlockSolve = 1u, kBlockInertFirst = 2u, kBlockInertSecond = 4u, kBlockPosition = 8u;
__device__ __forceinline__ bool block_supported(const TapeView& t, uint32_t s, uint32_t i) {
    const float4 mat = t.mat[t.cs(s) + i];
    return mat.z <= 0.0f && mat.x == 0.0f && mat.y == 0.0f;
}

// ---- forward: tape snapshots (run only inside a taped step) ----
__global__ void k_tape_clear_relay(TapeView t) {
    const uint32_t s = *t.slot;
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 4 * t.c; i += (size_t)gridDim.x * blockDim.x)
        t.relay[t.ps(s) + i] = kNoRelay;
}
// The step's contact set once its target speeds and relayed impulses are in place.
__global__ void k_tape_contacts(DeviceWorld w, TapeView t) {
    const uint32_t s = *t.slot;
    const uint32_t count = w.ctl[CTL_CONTACTS];
    if (blockIdx.x == 0 && threadIdx.x == 0) t.counts[s] = count;
    GRID_STRIDE(i, count) {
        const size_t o = t.cs(s) + i;
        t.rows[o] = w.cur.rows[i];
        t.normal[o] = w.cur.normal[i];
        t.mat[o] = w.cur.mat[i];
        t.ids[o] = w.cur.ids[i];
        t.extra[o] = w.cur.extra[i];
        for (uint32_t p = 0; p < 4u; ++p) {
            const size_t src = (size_t)p * w.c_cap + i;
            const size_t dst = t.ps(s) + (size_t)p * t.c + i;
            t.la[dst] = w.cur.la[src];
            t.lb[dst] = w.cur.lb[src];
            t.pos[dst] = w.cur.pos[src];
        }
    }
}
__global__ void k_tape_hot(DeviceWorld w, TapeView t, uint32_t k) {
    const uint32_t s = *t.slot;
    BodyHot* dst = t.hot + ((size_t)s * (t.substeps + 1) + k) * t.n;
    GRID_STRIDE(i, w.n) dst[i] = w.hot[i];
}
__global__ void k_tape_advance(TapeView t) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *t.slot += 1u;
}

// ---- backward ----
// Takes the slot below the counter; clears the per-step accumulators and the previous step's
// impulse gradient buffer (the relay fills it).
__global__ void k_adj_begin(TapeView t, AdjView a) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *t.slot -= 1u;
}
__global__ void k_adj_clear(TapeView t, AdjView a, uint32_t n) {
    const uint32_t s = *t.slot;
    const uint32_t count = t.counts[s];
    float4* prev = a.gacc[(*a.acc_flip) ^ 1u];
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 4 * t.c; i += (size_t)gridDim.x * blockDim.x) prev[i] = z;
    GRID_STRIDE(i, max(count, n)) {
        if (i < count) {
            for (uint32_t p = 0; p < 4u; ++p) {
                const size_t o = (size_t)p * t.c + i;
                a.g_ra[o] = z;
                a.g_rb[o] = z;
                a.g_m[o] = make_float2(0.0f, 0.0f);
                a.g_pt[o] = z;
            }
            a.g_param[i] = z;
            a.g_mu[i] = 0.0f;
        }
        if (i < n) {
            a.gres[i] = z;
            a.gres_acc[i] = z;
        }
    }
}

// Position iteration `it` of substep `k`, the row half: folds the contact contributions of the
// iteration reversed before (`fold`), then, unless it is past the first iteration (`it` valid),
// forms the gradient of the iteration's summed row delta (position_apply.wgsl:12-27 adds it, over
// the row's contribution count, to the position and to the resolution) and reverses the
// orientation's renormalisation.
__global__ void k_adj_prow(TapeView t, AdjView a, uint32_t n, uint32_t k, uint32_t it, bool fold, bool valid) {
    const uint32_t s = *t.slot;
    const BodyHot* start = t.hot_at(s, k);
    const BodyHot* end = t.hot_at(s, k + 1);
    GRID_STRIDE(i, n) {
        if (fold) {
            const float4 acc = a.gres_acc[i];
            const float4 g = a.gres[i];
            a.gres[i] = make_float4(g.x + acc.x, g.y + acc.y, g.z + acc.z, 0.0f);
            a.gres_acc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        if (!valid) continue;
        // a row no contact block claimed (aux.z) has no count on the tape and moved in no iteration
        const uint32_t cnt = start[i].aux.z == 0u ? 0u : t.cnt[t.pslot(s, k, it) + i];
        const BodyHot& h = end[i];
        if (cnt == 0u || !row_live(h)) {
            a.gsum[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            continue;
        }
        const f3 g = xyz(a.gx[i]) + xyz(a.gres[i]);
        a.gsum[i] = mk4(g / (float)cnt, 0.0f);
        // q' = normalize(q) with q unit to rounding: d q' / d q = I - q' q'^T
        const float4 q = h.rot;
        const float4 gq = a.gq[i];
        const float d = dot4(q, gq);
        a.gq[i] = make_float4(gq.x - q.x * d, gq.y - q.y * d, gq.z - q.z * d, gq.w - q.w * d);
    }
}
// The contact half: position_block's correction of each contact, reversed.
__global__ void k_adj_pcontact(TapeView t, AdjView a, dyn_step_params p, uint32_t k, uint32_t it) {
    const uint32_t s = *t.slot;
    const uint32_t count = t.counts[s];
    const BodyHot* hot = t.hot_at(s, k);
    const float4* res = t.res + t.pslot(s, k, it);
    GRID_STRIDE(i, count) {
        const uint32_t flags = __float_as_uint(a.t_tan2[i].w);
        if (!(flags & kBlockPosition)) continue;
        const uint4 r = t.rows[t.cs(s) + i];
        // a live row's inverse mass, 0 for an inert one (k_adj_terms, from the same rows; the blocks
        // the velocity iterations do not reverse read theirs)
        float ima, imb;
        if (flags & kBlockSolve) {
            const float4 body = a.t_body[i];
            ima = body.x;
            imb = body.y;
        } else {
            const BodyHot& ha = hot[r.x];
            const BodyHot& hb = hot[r.y];
            ima = row_live(ha) ? ha.pos.w : 0.0f;
            imb = row_live(hb) ? hb.pos.w : 0.0f;
        }
        const f3 normal = xyz(t.normal[t.cs(s) + i]);
        const float resolved = dot(normal, xyz(res[r.y]) - xyz(res[r.x]));
        const uint32_t pc = r.z & 0xFFu;
        f3 total = s3(0.0f);
        uint32_t contributing = 0;
        float error[4];
        const float kk = ima + imb;
        for (uint32_t q = 0; q < pc; ++q) {
            error[q] = wmax(t.la[t.ps(s) + (size_t)q * t.c + i].w - p.slop - resolved, 0.0f);
            if (error[q] <= 0.0f || kk == 0.0f) continue;
            total = total + normal * (p.relaxation * error[q] / kk);
            contributing += 1;
        }
        if (contributing == 0u) continue;
        const f3 correction = total / (float)contributing;
        const f3 la = -correction * ima;
        const f3 lb = correction * imb;
        if (!(dot(la, la) > 0.0f || dot(lb, lb) > 0.0f)) continue;
        const f3 g_la = ima > 0.0f ? xyz(a.gsum[r.x]) : s3(0.0f);
        const f3 g_lb = imb > 0.0f ? xyz(a.gsum[r.y]) : s3(0.0f);
        const f3 g_corr = imb * g_lb - ima * g_la;
        float g_ima = -dot(correction, g_la), g_imb = dot(correction, g_lb);
        const f3 g_total = g_corr / (float)contributing;
        const float gn = dot(normal, g_total);
        float g_resolved = 0.0f, g_k = 0.0f;
        for (uint32_t q = 0; q < pc; ++q) {
            if (error[q] <= 0.0f || kk == 0.0f) continue;
            const float g_err = p.relaxation / kk * gn;
            g_k += -p.relaxation * error[q] / (kk * kk) * gn;
            a.g_pt[(size_t)q * t.c + i].y += g_err;
            g_resolved -= g_err;
        }
        g_ima += g_k;
        g_imb += g_k;
        if (ima > 0.0f) atomic_add3(&a.gres_acc[r.x], -(normal * g_resolved));
        if (imb > 0.0f) atomic_add3(&a.gres_acc[r.y], normal * g_resolved);
        float4 gp = a.g_param[i];
        a.g_param[i] = make_float4(gp.x + g_ima, gp.y + g_imb, gp.z, gp.w);
    }
}

// substep_advance.wgsl:6-13 reversed: x' = x + v h; q' = normalize(q + h/2 (w, 0) q).
__global__ void k_adj_advance(TapeView t, AdjView a, uint32_t n, dyn_step_params p, uint32_t k) {
    const uint32_t s = *t.slot;
    const BodyHot* start = t.hot_at(s, k);
    const BodyHot* end = t.hot_at(s, k + 1);
    const float h = p.substep_dt;
    GRID_STRIDE(i, n) {
        const BodyHot& b = start[i];
        if (!row_live(b)) continue;
        const f3 gx = xyz(a.gx[i]);
        float4 gv = a.gv[i];
        a.gv[i] = make_float4(gv.x + h * gx.x, gv.y + h * gx.y, gv.z + h * gx.z, 0.0f);
        const float4 q = b.rot;
        const f3 w = xyz(end[i].ang);
        const float4 spin = make_float4(w.x, w.y, w.z, 0.0f);
        const float4 pq = add4(q, scale4(0.5f * h, quat_mul(spin, q)));
        const float len = sqrtf(dot4(pq, pq));
        const float4 qn = make_float4(pq.x / len, pq.y / len, pq.z / len, pq.w / len);
        const float4 gq = a.gq[i];
        const float d = dot4(qn, gq);
        const float4 gp = make_float4((gq.x - qn.x * d) / len, (gq.y - qn.y * d) / len, (gq.z - qn.z * d) / len,
                                      (gq.w - qn.w * d) / len);
        const f3 u = xyz(q), gpv = xyz(gp);
        const f3 gu = gpv + 0.5f * h * (cross(gpv, w) - gp.w * w);
        const float gs = gp.w + 0.5f * h * dot(gpv, w);
        a.gq[i] = mk4(gu, gs);
        const f3 gw = 0.5f * h * (q.w * gpv + cross(u, gpv) - gp.w * u);
        const float4 old = a.gw[i];
        a.gw[i] = make_float4(old.x + gw.x, old.y + gw.y, old.z + gw.z, 0.0f);
    }
}

// The pose-only terms of substep `k`'s contact blocks (k_solve_prepare's), once for all of the
// substep's reversed iterations.
// Also the block's flags and its bodies' inverse masses and inverse inertia scalars (isotropic bodies:
// the world inverse inertia is that scalar times the identity), so that the iterations read no body rows.
__global__ void k_adj_terms(TapeView t, AdjView a, uint32_t k) {
    const uint32_t s = *t.slot;
    const uint32_t count = t.counts[s];
    GRID_STRIDE(i, count) {
        const uint4 r = t.rows[t.cs(s) + i];
        uint32_t flags = 0u;
        if (resolves(r) && t.mat[t.cs(s) + i].z <= 0.0f) flags |= kBlockPosition;
        if (!resolves(r)) {
            a.t_tan2[i] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(flags));
            continue;
        }
        if (!block_supported(t, s, i)) {
            atomicOr(a.status, DYN_STATUS_ADJOINT_UNSUPPORTED);
            a.t_tan2[i] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(flags));
            continue;
        }
        TapeBlock b;
        tape_block(t, s, k, i, r, nullptr, &b);
        if (!(b.inert_f && b.inert_s)) flags |= kBlockSolve;
        if (b.inert_f) flags |= kBlockInertFirst;
        if (b.inert_s) flags |= kBlockInertSecond;
        a.t_body[i] = make_float4(b.pf.inverse_mass, b.ps.inverse_mass, b.pf.ii0.x, b.ps.ii0.x);
        a.t_tan1[i] = mk4(b.t1, 0.0f);
        a.t_tan2[i] = mk4(b.t2, __uint_as_float(flags));
#pragma unroll
        for (uint32_t q = 0; q < 4u; ++q) if (q < b.count) {
            const size_t o = (size_t)q * t.c + i;
            a.t_arm_a[o] = mk4(b.ra[q], b.nm[q]);
            a.t_arm_b[o] = mk4(b.rb[q], 0.0f);
            a.t_mass[o] = make_float4(b.m1[q], b.m2[q], t.lb[t.ps(s) + o].w, 0.0f);
        }
    }
}
// The block's bodies with the terms k_adj_terms stored.
__device__ __forceinline__ void tape_block_stored(const TapeView& t, const AdjView& a, uint32_t s, uint32_t k, uint32_t i,
                                                  uint4 r, const float4* vel, TapeBlock* b) {
    tape_block_bodies(t, s, k, i, r, vel, b);
    b->t1 = xyz(a.t_tan1[i]);
    b->t2 = xyz(a.t_tan2[i]);
#pragma unroll
    for (uint32_t q = 0; q < 4u; ++q) if (q < b->count) {
        const size_t o = (size_t)q * t.c + i;
        const float4 x = a.t_arm_a[o], y = a.t_arm_b[o], m = a.t_mass[o];
        b->ra[q] = xyz(x);
        b->nm[q] = x.w;
        b->rb[q] = xyz(y);
        b->m1[q] = m.x;
        b->m2[q] = m.y;
    }
}

// One contact block of velocity iteration `it` of substep `k` (solve_block of step.cuh), reversed.
// Every point's impulse comes from the velocities the block started with, so each point reverses on
// its own: a quad of lanes takes a block, one point per lane, and sums the block's velocity and
// parameter gradients over the quad with shuffles; the quad's first lane adds them to the rows.
__device__ __forceinline__ float quad_sum(float v, unsigned mask) {
    v += __shfl_xor_sync(mask, v, 1);
    v += __shfl_xor_sync(mask, v, 2);
    return v;
}
__device__ __forceinline__ f3 quad_sum3(f3 v, unsigned mask) {
    return mk3(quad_sum(v.x, mask), quad_sum(v.y, mask), quad_sum(v.z, mask));
}
__global__ void __launch_bounds__(128, 6) k_adj_solve(TapeView t, AdjView a, dyn_step_params p, uint32_t k, uint32_t it) {
    const uint32_t s = *t.slot;
    const uint32_t count = t.counts[s];
    const float4* vel = t.vel_at(s, k, it);
    const float4* accs = t.acc_at(s, k, it);
    float4* gacc = a.gacc[*a.acc_flip];
    const uint32_t q = threadIdx.x & 3u;  // the lane's point
    const unsigned mask = 0xFu << (threadIdx.x & 28u);
    const uint32_t quads = (gridDim.x * blockDim.x) >> 2;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 2; i < count; i += quads) {
        // every lane of a quad takes the same branches up to the point work. Everything that does not
        // depend on the block's rows is loaded first, in one round trip (the point arrays hold 4c
        // entries, so every lane's loads are in bounds whatever the block's point count)
        const float4 tan2 = a.t_tan2[i];
        const uint4 r = t.rows[t.cs(s) + i];
        const float4 body = a.t_body[i];
        const float4 nf = t.normal[t.cs(s) + i];
        const float4 tan1 = a.t_tan1[i];
        const size_t o = (size_t)q * t.c + i;
        const float4 arm_a = a.t_arm_a[o], arm_b = a.t_arm_b[o], masses = a.t_mass[o];
        const float4 acc = accs[o];
        const float4 gout = gacc[o];
        const float4 gra0 = a.g_ra[o], grb0 = a.g_rb[o];
        const float2 gm0 = a.g_m[o];
        const uint32_t flags = __float_as_uint(tan2.w);
        if (!(flags & kBlockSolve)) continue;
        const bool inert_f = (flags & kBlockInertFirst) != 0u, inert_s = (flags & kBlockInertSecond) != 0u;
        const float ima = body.x, imb = body.y;
        // the bodies as the block saw them: only the velocities are read (dbody_iinv of an isotropic
        // body is its scalar times the vector)
        DBody pf, ps;
        pf.velocity = xyz(vel[r.x]);
        pf.angular_velocity = xyz(vel[t.n + r.x]);
        ps.velocity = xyz(vel[r.y]);
        ps.angular_velocity = xyz(vel[t.n + r.y]);
        const f3 dva = inert_f ? s3(0.0f) : xyz(a.gv[r.x]);
        const f3 dwa = inert_f ? s3(0.0f) : xyz(a.gw[r.x]);
        const f3 dvb = inert_s ? s3(0.0f) : xyz(a.gv[r.y]);
        const f3 dwb = inert_s ? s3(0.0f) : xyz(a.gw[r.y]);
        const f3 Wa = dwa * body.z;
        const f3 Wb = dwb * body.w;
        f3 bva = s3(0.0f), bwa = s3(0.0f), bvb = s3(0.0f), bwb = s3(0.0f);
        float g_ima = 0.0f, g_imb = 0.0f, g_sa = 0.0f, g_sb = 0.0f, g_mu = 0.0f;
        if (q < (r.z & 0xFFu)) {
            const f3 n = xyz(nf), t1 = xyz(tan1), t2 = xyz(tan2);
            const float mu = nf.w;
            const f3 ra = xyz(arm_a), rb = xyz(arm_b);
            const float nm = arm_a.w, m1 = masses.x, m2 = masses.y, target = masses.z;
            const float an = acc.x, at1 = acc.y, at2 = acc.z;
            // forward (solve_block, hard contact)
            const f3 rel = point_velocity_arm(ps, rb) - point_velocity_arm(pf, ra);
            const float ns = dot(rel, n);
            const float delta = (target - ns) / nm;
            const float an1 = wmax(0.0f, an + delta);
            const float lim = mu * an1;
            const float ts1 = dot(rel, t1);
            const float u1 = at1 - ts1 / m1;
            const float at11 = wclamp(u1, -lim, lim);
            const float ts2 = dot(rel, t2);
            const float rem2 = lim * lim - at11 * at11;
            const float rem = sqrtf(wmax(rem2, 0.0f));
            const float u2 = at2 - ts2 / m2;
            const float at21 = wclamp(u2, -rem, rem);
            const f3 j = s3(0.0f) + n * (an1 - an) + t1 * (at11 - at1) + t2 * (at21 - at2);
            // reverse: the impulse's effect on both bodies
            const f3 jb = imb * dvb - ima * dva + cross(ra, Wa) + cross(Wb, rb);
            g_ima = -dot(dva, j);
            g_imb = dot(dvb, j);
            g_sa = -dot(Wa, cross(ra, j));
            g_sb = dot(Wb, cross(rb, j));
            f3 gra = cross(Wa, j), grb = cross(j, Wb);
            float g_an1 = dot(n, jb) + gout.x, g_an0 = -dot(n, jb);
            float g_at11 = dot(t1, jb) + gout.y, g_at10 = -dot(t1, jb);
            const float g_at21 = dot(t2, jb) + gout.z;
            float g_at20 = -dot(t2, jb);
            // at2' = clamp(u2, -rem, rem)
            float g_u2 = 0.0f, g_rem = 0.0f;
            if (u2 > rem) {
                g_rem += g_at21;
            } else if (u2 < -rem) {
                g_rem -= g_at21;
            } else {
                g_u2 = g_at21;
            }
            g_at20 += g_u2;
            const float g_ts2 = -g_u2 / m2;
            const float g_m2 = g_u2 * ts2 / (m2 * m2);
            float g_lim = 0.0f;
            if (rem2 > 0.0f && rem > kTangentLimitFloor * lim) {
                const float g_rem2 = 0.5f * g_rem / rem;
                g_lim += 2.0f * lim * g_rem2;
                g_at11 -= 2.0f * at11 * g_rem2;
            }
            // at1' = clamp(u1, -lim, lim)
            float g_u1 = 0.0f;
            if (u1 > lim) {
                g_lim += g_at11;
            } else if (u1 < -lim) {
                g_lim -= g_at11;
            } else {
                g_u1 = g_at11;
            }
            g_at10 += g_u1;
            const float g_ts1 = -g_u1 / m1;
            const float g_m1 = g_u1 * ts1 / (m1 * m1);
            // lim = mu an'
            g_an1 += mu * g_lim;
            g_mu = an1 * g_lim;
            // an' = max(0, an + delta)
            float g_delta = 0.0f;
            if (an + delta > 0.0f) {
                g_an0 += g_an1;
                g_delta = g_an1;
            }
            // delta = (target - ns) / nm
            const float g_target = g_delta / nm;
            const float g_ns = -g_delta / nm;
            const float g_nm = -g_delta * delta / nm;
            const f3 g_rel = n * g_ns + t1 * g_ts1 + t2 * g_ts2;
            bvb = g_rel;
            bva = -g_rel;
            bwb = cross(rb, g_rel);
            bwa = -cross(ra, g_rel);
            grb = grb + cross(g_rel, ps.angular_velocity);
            gra = gra - cross(g_rel, pf.angular_velocity);
            gacc[o] = make_float4(g_an0, g_at10, g_at20, 0.0f);
            a.g_ra[o] = make_float4(gra0.x + gra.x, gra0.y + gra.y, gra0.z + gra.z, gra0.w + g_nm);
            a.g_rb[o] = make_float4(grb0.x + grb.x, grb0.y + grb.y, grb0.z + grb.z, grb0.w + g_target);
            a.g_m[o] = make_float2(gm0.x + g_m1, gm0.y + g_m2);
        }
        bva = quad_sum3(bva, mask);
        bwa = quad_sum3(bwa, mask);
        bvb = quad_sum3(bvb, mask);
        bwb = quad_sum3(bwb, mask);
        g_ima = quad_sum(g_ima, mask);
        g_imb = quad_sum(g_imb, mask);
        g_sa = quad_sum(g_sa, mask);
        g_sb = quad_sum(g_sb, mask);
        g_mu = quad_sum(g_mu, mask);
        if (q == 0u) {
            if (!inert_f) {
                atomic_add3(&a.gv_acc[r.x], bva);
                atomic_add3(&a.gw_acc[r.x], bwa);
            }
            if (!inert_s) {
                atomic_add3(&a.gv_acc[r.y], bvb);
                atomic_add3(&a.gw_acc[r.y], bwb);
            }
            const float4 gp = a.g_param[i];
            a.g_param[i] = make_float4(gp.x + g_ima, gp.y + g_imb, gp.z + g_sa, gp.w + g_sb);
            a.g_mu[i] += g_mu;
        }
    }
}
// solver_block_apply.wgsl reversed: v' = v + sum of the blocks' changes.
__global__ void k_adj_vmerge(AdjView a, uint32_t n) {
    GRID_STRIDE(i, n) {
        const float4 dv = a.gv_acc[i], dw = a.gw_acc[i];
        const float4 v = a.gv[i], w = a.gw[i];
        a.gv[i] = make_float4(v.x + dv.x, v.y + dv.y, v.z + dv.z, 0.0f);
        a.gw[i] = make_float4(w.x + dw.x, w.y + dw.y, w.z + dw.z, 0.0f);
        a.gv_acc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        a.gw_acc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}
// The warm start of substep 0 (solver_contact_block.wgsl:195-233) reversed: its velocity changes do
// not depend on the velocities, only on the relayed impulses, the arms and the masses.
__global__ void k_adj_warm(TapeView t, AdjView a) {
    const uint32_t s = *t.slot;
    const uint32_t count = t.counts[s];
    float4* gacc = a.gacc[*a.acc_flip];
    GRID_STRIDE(i, count) {
        const uint4 r = t.rows[t.cs(s) + i];
        if (!resolves(r) || !block_supported(t, s, i)) continue;
        TapeBlock b;
        tape_block_stored(t, a, s, 0, i, r, nullptr, &b);
        if (b.inert_f && b.inert_s) continue;
        const f3 dva = b.inert_f ? s3(0.0f) : xyz(a.gv[r.x]);
        const f3 dwa = b.inert_f ? s3(0.0f) : xyz(a.gw[r.x]);
        const f3 dvb = b.inert_s ? s3(0.0f) : xyz(a.gv[r.y]);
        const f3 dwb = b.inert_s ? s3(0.0f) : xyz(a.gw[r.y]);
        const f3 Wa = dbody_iinv(b.pf, dwa);
        const f3 Wb = dbody_iinv(b.ps, dwb);
        const float ima = b.pf.inverse_mass, imb = b.ps.inverse_mass;
        const float4* accs = t.acc_at(s, 0, 0);  // the warm start leaves the impulses as iteration 0 finds them
        float g_ima = 0.0f, g_imb = 0.0f, g_sa = 0.0f, g_sb = 0.0f;
        #pragma unroll
        for (uint32_t q = 0; q < 4u; ++q) if (q < b.count) {
            const size_t o = (size_t)q * t.c + i;
            const float4 acc = accs[o];
            const f3 j = b.normal * acc.x + b.t1 * acc.y + b.t2 * acc.z;
            const f3 jb = imb * dvb - ima * dva + cross(b.ra[q], Wa) + cross(Wb, b.rb[q]);
            const float4 g = gacc[o];
            gacc[o] = make_float4(g.x + dot(b.normal, jb), g.y + dot(b.t1, jb), g.z + dot(b.t2, jb), 0.0f);
            g_ima -= dot(dva, j);
            g_imb += dot(dvb, j);
            g_sa -= dot(Wa, cross(b.ra[q], j));
            g_sb += dot(Wb, cross(b.rb[q], j));
            const f3 gra = cross(Wa, j), grb = cross(j, Wb);
            float4 x = a.g_ra[o];
            a.g_ra[o] = make_float4(x.x + gra.x, x.y + gra.y, x.z + gra.z, x.w);
            x = a.g_rb[o];
            a.g_rb[o] = make_float4(x.x + grb.x, x.y + grb.y, x.z + grb.z, x.w);
        }
        const float4 gp = a.g_param[i];
        a.g_param[i] = make_float4(gp.x + g_ima, gp.y + g_imb, gp.z + g_sa, gp.w + g_sb);
    }
}
// k_solve_prepare reversed for substep `k`: the arm and effective-mass gradients the substep's warm
// start and iterations collected become orientation gradients (arm = R (anchor - centre of mass))
// and inverse mass / inertia scale gradients; then they are cleared for the substep before.
__global__ void k_adj_prepare(TapeView t, AdjView a, uint32_t k) {
    const uint32_t s = *t.slot;
    const uint32_t count = t.counts[s];
    GRID_STRIDE(i, count) {
        const uint4 r = t.rows[t.cs(s) + i];
        if (!resolves(r) || !block_supported(t, s, i)) continue;
        TapeBlock b;
        tape_block(t, s, k, i, r, nullptr, &b);
        if (b.inert_f && b.inert_s) continue;
        const f3 n = b.normal;
        float g_sim_a = 0.0f, g_sim_b = 0.0f, g_ssc_a = 0.0f, g_ssc_b = 0.0f;
        f3 g_spread_f = s3(0.0f), g_spread_s = s3(0.0f);
        f3 gra[4], grb[4];
        #pragma unroll
        for (uint32_t q = 0; q < 4u; ++q) if (q < b.count) {
            const size_t o = (size_t)q * t.c + i;
            const float4 xa = a.g_ra[o], xb = a.g_rb[o];
            const float2 xm = a.g_m[o];
            gra[q] = xyz(xa);
            grb[q] = xyz(xb);
            const f3 ra = b.ra[q], rb = b.rb[q];
            // normal mass = count (split im_a + split im_b) + spread_f . (ra x n) + spread_s . (rb x n)
            const float g_nm = xa.w;
            g_sim_a += b.count_f * g_nm;
            g_sim_b += b.count_f * g_nm;
            g_spread_f = g_spread_f + cross(ra, n) * g_nm;
            g_spread_s = g_spread_s + cross(rb, n) * g_nm;
            gra[q] = gra[q] + cross(n, b.spread_f * g_nm);
            grb[q] = grb[q] + cross(n, b.spread_s * g_nm);
            // tangent masses = count (split im_a + split im_b + (ra x t).S_a(ra x t) + (rb x t).S_b(rb x t))
            for (int axis = 0; axis < 2; ++axis) {
                const f3 tt = axis == 0 ? b.t1 : b.t2;
                const float g = (axis == 0 ? xm.x : xm.y) * b.count_f;
                const f3 rax = cross(ra, tt), rbx = cross(rb, tt);
                const f3 sa = dbody_iinv(b.sf, rax), sb = dbody_iinv(b.ss, rbx);
                g_sim_a += g;
                g_sim_b += g;
                gra[q] = gra[q] + cross(tt, sa * (2.0f * g));
                grb[q] = grb[q] + cross(tt, sb * (2.0f * g));
                g_ssc_a += g * dot(rax, sa);
                g_ssc_b += g * dot(rbx, sb);
            }
            a.g_ra[o] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            a.g_rb[o] = make_float4(0.0f, 0.0f, 0.0f, xb.w);  // the target speed's gradient stays for the step's start
            a.g_m[o] = make_float2(0.0f, 0.0f);
        }
        // spread = S_split (reach x n): reach = sum of the arms
        const f3 gxf = dbody_iinv(b.sf, g_spread_f), gxs = dbody_iinv(b.ss, g_spread_s);
        const f3 g_reach_f = cross(n, gxf), g_reach_s = cross(n, gxs);
        g_ssc_a += dot(g_spread_f, b.spread_f);
        g_ssc_b += dot(g_spread_s, b.spread_s);
        // arm = (R la + x) - (x + R com): only the orientation moves it
        const float count_a = (float)max(t.hot_at(s, k)[r.x].aux.z, 1u), count_b = (float)max(t.hot_at(s, k)[r.y].aux.z, 1u);
        float4 gqa = make_float4(0.0f, 0.0f, 0.0f, 0.0f), gqb = gqa;
        #pragma unroll
        for (uint32_t q = 0; q < 4u; ++q) if (q < b.count) {
            const size_t o = t.ps(s) + (size_t)q * t.c + i;
            const f3 ga = gra[q] + g_reach_f, gb = grb[q] + g_reach_s;
            gqa = add4(gqa, quat_rotate_qgrad(b.pf.orientation, xyz(t.la[o]) - b.pf.com, ga));
            gqb = add4(gqb, quat_rotate_qgrad(b.ps.orientation, xyz(t.lb[o]) - b.ps.com, gb));
        }
        if (!b.inert_f) atomic_add4(&a.gq[r.x], gqa);
        if (!b.inert_s) atomic_add4(&a.gq[r.y], gqb);
        // split inverse mass = count x inverse mass; the split tensor scales with the tensor
        const float4 gp = a.g_param[i];
        a.g_param[i] = make_float4(gp.x + count_a * g_sim_a, gp.y + count_b * g_sim_b, gp.z + g_ssc_a, gp.w + g_ssc_b);
    }
}
// substep_integrate.wgsl:15-76 reversed (no applied forces; isotropic bodies keep their spin):
// v' = clamp_speed(v + g h) / (1 + c h), w' = clamp_spin(w) / (1 + c_w h).
__global__ void k_adj_integrate(DeviceWorld w, TapeView t, AdjView a, dyn_step_params p, uint32_t k) {
    const uint32_t s = *t.slot;
    const BodyHot* start = t.hot_at(s, k);
    const float h = p.substep_dt;
    GRID_STRIDE(i, w.n) {
        const BodyHot& b = start[i];
        if (!row_live(b)) continue;
        const float4 dm = w.damp[i];
        const f3 velocity = xyz(b.vel) + mk3(p.gravity[0], p.gravity[1], p.gravity[2]) * dm.z * h;
        const f3 angular = xyz(b.ang);
        f3 gv = xyz(a.gv[i]) / (1.0f + dm.x * h);
        f3 gw = xyz(a.gw[i]) / (1.0f + dm.y * h);
        const float speed = length(velocity);
        if (speed > p.max_velocity) {
            const f3 u = velocity / speed;
            gv = (gv - u * dot(u, gv)) * (p.max_velocity / speed);
        }
        const float spin = length(angular);
        if (spin > p.max_angular_velocity) {
            const f3 u = angular / spin;
            gw = (gw - u * dot(u, gw)) * (p.max_angular_velocity / spin);
        }
        a.gv[i] = mk4(gv, 0.0f);
        a.gw[i] = mk4(gw, 0.0f);
    }
}
// The step's start, reversed: target speeds (solver_blocks.wgsl:24-48) and the depth of the frozen
// contacts move with the bodies' poses and velocities at the step's start; the relayed impulses'
// gradient goes to the previous step's points (contact_relay.wgsl:34-72); contact friction
// (combined from both colliders' frictions, narrowphase.wgsl) and the blocks' parameter gradients
// go to colliders and rows.
__global__ void k_adj_start(DeviceWorld w, TapeView t, AdjView a, dyn_step_params p) {
    const uint32_t s = *t.slot;
    const uint32_t count = t.counts[s];
    const BodyHot* start = t.hot_at(s, 0);
    const float4* gacc = a.gacc[*a.acc_flip];
    float4* gprev = a.gacc[(*a.acc_flip) ^ 1u];
    GRID_STRIDE(i, count) {
        const uint4 r = t.rows[t.cs(s) + i];
        const uint32_t pc = r.z & 0xFFu;
        for (uint32_t q = 0; q < pc; ++q) {
            const size_t o = (size_t)q * t.c + i;
            const uint32_t src = t.relay[t.ps(s) + o];
            if (src != kNoRelay) gprev[src] = gacc[o];
        }
        if (!resolves(r) || !block_supported(t, s, i)) continue;
        const BodyHot& ha = start[r.x];
        const BodyHot& hb = start[r.y];
        const bool live_a = row_live(ha), live_b = row_live(hb);
        const f3 n = xyz(t.normal[t.cs(s) + i]);
        const float restitution = t.extra[t.cs(s) + i].x;
        f3 gxa = s3(0.0f), gxb = s3(0.0f), gva = s3(0.0f), gvb = s3(0.0f), gwa = s3(0.0f), gwb = s3(0.0f);
        float4 gqa = make_float4(0.0f, 0.0f, 0.0f, 0.0f), gqb = gqa;
        const DBody fa = tape_body(ha, ha.vel, ha.ang), fb = tape_body(hb, hb.vel, hb.ang);
        for (uint32_t q = 0; q < pc; ++q) {
            const size_t o = (size_t)q * t.c + i;
            const float g_target = a.g_rb[o].w;
            const float depth = t.la[t.ps(s) + o].w;
            float g_depth = a.g_pt[o].y;
            if (depth < 0.0f) {
                g_depth += g_target / p.dt;
            } else {
                const f3 position = xyz(t.pos[t.ps(s) + o]);
                const f3 arm_a = position - dbody_com(fa), arm_b = position - dbody_com(fb);
                const float speed = dot(point_velocity_arm(fb, arm_b) - point_velocity_arm(fa, arm_a), n);
                if (speed < -p.restitution_threshold) {
                    const f3 g_rel = n * (-restitution * g_target);
                    gvb = gvb + g_rel;
                    gva = gva - g_rel;
                    gwb = gwb + cross(arm_b, g_rel);
                    gwa = gwa - cross(arm_a, g_rel);
                    // arm = point - (x + R com)
                    const f3 g_arm_b = cross(g_rel, fb.angular_velocity), g_arm_a = -cross(g_rel, fa.angular_velocity);
                    gxb = gxb - g_arm_b;
                    gxa = gxa - g_arm_a;
                    gqb = add4(gqb, scale4(-1.0f, quat_rotate_qgrad(fb.orientation, fb.com, g_arm_b)));
                    gqa = add4(gqa, scale4(-1.0f, quat_rotate_qgrad(fa.orientation, fa.com, g_arm_a)));
                }
            }
            // d = d0 + n . ((x_a + R_a la) - (x_b + R_b lb))
            const f3 g = n * g_depth;
            gxa = gxa + g;
            gxb = gxb - g;
            gqa = add4(gqa, quat_rotate_qgrad(fa.orientation, xyz(t.la[t.ps(s) + o]), g));
            gqb = add4(gqb, scale4(-1.0f, quat_rotate_qgrad(fb.orientation, xyz(t.lb[t.ps(s) + o]), g)));
        }
        if (live_a) {
            atomic_add3(&a.gx[r.x], gxa);
            atomic_add4(&a.gq[r.x], gqa);
            atomic_add3(&a.gv[r.x], gva);
            atomic_add3(&a.gw[r.x], gwa);
        }
        if (live_b) {
            atomic_add3(&a.gx[r.y], gxb);
            atomic_add4(&a.gq[r.y], gqb);
            atomic_add3(&a.gv[r.y], gvb);
            atomic_add3(&a.gw[r.y], gwb);
        }
        const float4 gp = a.g_param[i];
        if (live_a) {
            atomicAdd(&a.g_im[r.x], gp.x);
            atomicAdd(&a.g_scale[r.x], gp.z);
        }
        if (live_b) {
            atomicAdd(&a.g_im[r.y], gp.y);
            atomicAdd(&a.g_scale[r.y], gp.w);
        }
        // contact friction = combine(friction of collider a, of collider b), narrowphase's write_contact
        const float g_mu = a.g_mu[i];
        if (g_mu != 0.0f) {
            const uint4 ids = t.ids[t.cs(s) + i];
            const float fa_ = w.c_mat[ids.x].x, fb_ = w.c_mat[ids.y].x;
            float da = 0.0f, db = 0.0f;
            if (p.friction_combine == 1u) {
                (fa_ < fb_ ? da : db) = 1.0f;
            } else if (p.friction_combine == 2u) {
                (fa_ > fb_ ? da : db) = 1.0f;
            } else if (p.friction_combine == 3u) {
                da = db = 0.5f;
            } else {
                const float mu = sqrtf(fa_ * fb_);
                da = fa_ > 0.0f ? 0.5f * mu / fa_ : 0.0f;
                db = fb_ > 0.0f ? 0.5f * mu / fb_ : 0.0f;
            }
            atomicAdd(&a.g_friction[ids.x], g_mu * da);
            atomicAdd(&a.g_friction[ids.y], g_mu * db);
        }
    }
}
// The end of a reversed step: the previous step's impulse gradient becomes the current one.
__global__ void k_adj_end(AdjView a) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.acc_flip ^= 1u;
}

// Rows patched by a step's queued edits (body_edits.wgsl PATCH): the state before the edit has no
// influence on the patched fields, so their gradient stops there. masks[i] = DYN_PATCH_* bits of row rows[i].
__global__ void k_adj_patch(AdjView a, const uint32_t* rows, const uint32_t* masks, uint32_t m) {
    GRID_STRIDE(i, m) {
        const uint32_t row = rows[i], mask = masks[i];
        const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (mask & DYN_PATCH_POSITION) a.gx[row] = z;
        if (mask & DYN_PATCH_ORIENTATION) a.gq[row] = z;
        if (mask & DYN_PATCH_VELOCITY) a.gv[row] = z;
        if (mask & DYN_PATCH_ANGULAR_VELOCITY) a.gw[row] = z;
    }
}

__global__ void k_grad_unpack(AdjView a, const dyn_body_grad* __restrict__ in, uint32_t n) {
    GRID_STRIDE(i, n) {
        const dyn_body_grad& g = in[i];
        a.gx[i] = make_float4(g.position[0], g.position[1], g.position[2], 0.0f);
        a.gq[i] = make_float4(g.orientation[0], g.orientation[1], g.orientation[2], g.orientation[3]);
        a.gv[i] = make_float4(g.velocity[0], g.velocity[1], g.velocity[2], 0.0f);
        a.gw[i] = make_float4(g.angular_velocity[0], g.angular_velocity[1], g.angular_velocity[2], 0.0f);
    }
}
__global__ void k_grad_pack(AdjView a, dyn_body_grad* __restrict__ out, uint32_t n) {
    GRID_STRIDE(i, n) {
        dyn_body_grad g;
        const float4 x = a.gx[i], q = a.gq[i], v = a.gv[i], av = a.gw[i];
        g.position[0] = x.x; g.position[1] = x.y; g.position[2] = x.z; g._pad0 = 0.0f;
        g.orientation[0] = q.x; g.orientation[1] = q.y; g.orientation[2] = q.z; g.orientation[3] = q.w;
        g.velocity[0] = v.x; g.velocity[1] = v.y; g.velocity[2] = v.z; g._pad1 = 0.0f;
        g.angular_velocity[0] = av.x; g.angular_velocity[1] = av.y; g.angular_velocity[2] = av.z; g._pad2 = 0.0f;
        out[i] = g;
    }
}

// Parameters of a differentiable rollout onto the device rows and colliders (dyn_set_mass_properties,
// dyn_set_friction).
__global__ void k_set_mass(DeviceWorld w, const float* __restrict__ im, const float* __restrict__ ii,
                           const float* __restrict__ inertia, uint32_t n) {
    GRID_STRIDE(i, n) {
        BodyHot& h = w.hot[i];
        h.pos.w = im[i];
        const float* t = ii + 6 * (size_t)i;
        const float* I = inertia + 6 * (size_t)i;
        h.ii0 = make_float4(t[0], t[1], t[2], t[3]);
        h.ii1 = make_float4(t[4], t[5], 0.0f, 0.0f);
        w.inert0[i] = make_float4(I[0], I[1], I[2], I[3]);
        w.inert1[i] = make_float2(I[4], I[5]);
    }
}
__global__ void k_set_friction(DeviceWorld w, const float* __restrict__ friction, uint32_t k) {
    GRID_STRIDE(i, k) {
        const float4 m = w.c_mat[i];
        w.c_mat[i] = make_float4(friction[i], m.y, m.z, m.w);
    }
}

}  // namespace dyn
