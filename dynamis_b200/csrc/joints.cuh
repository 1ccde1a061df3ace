// joints.cuh - ball joints: the warm start, velocity and position passes, the jointed-pair filter
// and the island coupling of constraints.
//
// Joints are solved Gauss-Seidel within a component (a connected set of joints), layer by layer in
// the order of the host planner (plan_joints, crates/dynamis-world/src/schedule.rs:105-296), with a
// forward and a backward sweep per pass (joint_velocity.wgsl:24-54, joint_position.wgsl:30-61).
// The joints of one layer share no body, and components share none either, so a layer's joints run
// in parallel and components run independently. The device packs components into 32-lane warps
// (JointPlan::groups): a component owns `lanes` lanes, steps through its layers, and the warp meets
// at __syncwarp after every layer, which also orders the body rows one layer writes before the next
// layer reads them. Body rows are read and written in place, as the reference's joint passes do:
// these passes run as kernels of their own, between the contact kernels of the same iteration.
#pragma once

#include "step.cuh"

namespace dyn {

enum JointPass : int { JP_WARM = 0, JP_SOLVE = 1, JP_POSITION = 2 };

struct JointForces {  // FrameForces (joint_solve.wgsl:1-6)
    f3 linear_first, angular_first, linear_second, angular_second;
};

__device__ __forceinline__ void store_velocities(const DeviceWorld& w, uint32_t row, const DBody& b) {
    w.hot[row].vel = mk4(b.velocity, 0.0f);
    w.hot[row].ang = mk4(b.angular_velocity, 0.0f);
}

// joint_solve.wgsl:803-832 (warm_joint) for a ball joint (warm_constraint_rows :754-766).
__device__ __forceinline__ void joint_warm(const DeviceWorld& w, uint32_t j) {
    const dyn_constraint_runtime_record& rt = w.jruntime[j];
    if (rt.broken != 0u) return;
    const uint4 meta = w.jmeta[j];
    DBody fl = load_dbody(w.hot, meta.z), sl = load_dbody(w.hot, meta.w);
    DBody first = dbody_inert(fl) ? dbody_frozen(fl) : fl;
    DBody second = dbody_inert(sl) ? dbody_frozen(sl) : sl;
    if (meta.y & DYN_CONSTRAINT_WARM_START) {
        f3 anchor_a = arm(first, xyz(w.janchor_a[j]));
        f3 anchor_b = arm(second, xyz(w.janchor_b[j]));
        for (uint32_t i = 0; i < 3; ++i) {
            f3 axis = mk3(i == 0 ? 1.0f : 0.0f, i == 1 ? 1.0f : 0.0f, i == 2 ? 1.0f : 0.0f);
            pair_impulse(&first, &second, anchor_a, anchor_b, axis * rt.accumulated[i]);
        }
    }
    store_velocities(w, meta.z, first);
    store_velocities(w, meta.w, second);
}

// joint_solve.wgsl:236-267 and 419-430 (solve_joint for a ball joint: three point rows along the
// world axes, solve_point_row :96-128), then the break test (:679-686) and the write-back.
__device__ __forceinline__ void joint_solve(const DeviceWorld& w, const dyn_step_params& p, uint32_t j, bool residual) {
    dyn_constraint_runtime_record& rt = w.jruntime[j];
    const uint4 meta = w.jmeta[j];
    const bool warm = (meta.y & DYN_CONSTRAINT_WARM_START) != 0u;
    if (rt.broken != 0u) return;
    DBody fl = load_dbody(w.hot, meta.z), sl = load_dbody(w.hot, meta.w);
    if (dbody_inert(fl) && dbody_inert(sl)) return;
    DBody first = dbody_inert(fl) ? dbody_frozen(fl) : fl;
    DBody second = dbody_inert(sl) ? dbody_frozen(sl) : sl;
    const DBody mass_first = first, mass_second = second;
    const float4 aa4 = w.janchor_a[j], ab4 = w.janchor_b[j];
    const f3 anchor_a = arm(first, xyz(aa4));
    const f3 anchor_b = arm(second, xyz(ab4));
    float acc[3];
    for (uint32_t i = 0; i < 3; ++i) acc[i] = warm ? rt.accumulated[i] : 0.0f;
    JointForces f{s3(0.0f), s3(0.0f), s3(0.0f), s3(0.0f)};
    for (uint32_t i = 0; i < 3; ++i) {
        const f3 axis = mk3(i == 0 ? 1.0f : 0.0f, i == 1 ? 1.0f : 0.0f, i == 2 ? 1.0f : 0.0f);
        const float k = momentum_mass(mass_first, mass_second, anchor_a, anchor_b, axis);
        if (k > 0.0f) {
            const DBody before_first = first, before_second = second;
            const float speed = dot(relative_velocity(first, second, anchor_a, anchor_b), axis);
            const float next = acc[i] - speed / k;
            const float applied = next - acc[i];  // row_impulse with no cap
            pair_impulse(&first, &second, anchor_a, anchor_b, axis * applied);
            acc[i] = next;
            // point_reaction (joint_solve.wgsl:58-69) over the bodies the row started from
            const f3 impulse = axis * acc[i];
            f.linear_first = f.linear_first + (-impulse);
            f.linear_second = f.linear_second + impulse;
            f.angular_first = f.angular_first + cross(anchor_a - dbody_com(before_first), -impulse);
            f.angular_second = f.angular_second + cross(anchor_b - dbody_com(before_second), impulse);
        }
    }
    uint32_t broken = 0u;
    if (meta.y & DYN_CONSTRAINT_HAS_BREAK) {
        const float force = length(f.linear_second) / p.dt;
        const float torque = length(f.angular_second) / p.dt;
        if ((aa4.w > 0.0f && force > aa4.w) || (ab4.w > 0.0f && torque > ab4.w)) broken = 1u;
    }
    for (uint32_t i = 0; i < 3; ++i) rt.accumulated[i] = acc[i];
    if (!warm) {
        for (uint32_t i = 3; i < DYN_CONSTRAINT_ACCUMULATOR_SLOTS; ++i) rt.accumulated[i] = 0.0f;
    }
    dyn_constraint_reaction_record& rx = rt.reaction;
    rx.linear_first[0] = f.linear_first.x; rx.linear_first[1] = f.linear_first.y; rx.linear_first[2] = f.linear_first.z;
    rx.angular_first[0] = f.angular_first.x; rx.angular_first[1] = f.angular_first.y; rx.angular_first[2] = f.angular_first.z;
    rx.linear_second[0] = f.linear_second.x; rx.linear_second[1] = f.linear_second.y; rx.linear_second[2] = f.linear_second.z;
    rx.angular_second[0] = f.angular_second.x; rx.angular_second[1] = f.angular_second.y;
    rx.angular_second[2] = f.angular_second.z;
    rx._pad_linear_first = rx._pad_angular_first = rx._pad_linear_second = rx._pad_angular_second = 0.0f;
    if (broken) rt.broken = 1u;
    store_velocities(w, meta.z, first);
    store_velocities(w, meta.w, second);
    if (residual) {
        max_counter(&w.counters[DYN_COUNTER_SOLVE_LINEAR_RESIDUAL],
                    (uint32_t)solver_word(wmax(length(first.velocity - fl.velocity), length(second.velocity - sl.velocity)),
                                          DYN_SOLVER_VELOCITY_SCALE));
        max_counter(&w.counters[DYN_COUNTER_SOLVE_ANGULAR_RESIDUAL],
                    (uint32_t)solver_word(wmax(length(first.angular_velocity - fl.angular_velocity),
                                               length(second.angular_velocity - sl.angular_velocity)),
                                          DYN_SOLVER_VELOCITY_SCALE));
    }
}

// correction.wgsl:32-35 (apply_correction) for a purely linear correction.
__device__ __forceinline__ void shift_body(DBody* b, f3 linear, f3 angular) {
    b->position = b->position + linear;
    b->orientation = normalize4(quat_mul(mk4(angular * 0.5f, 1.0f), b->orientation));
}

// joint_position.wgsl:18-36 (project) over joint_correction.wgsl:5-27, 85-90 for a ball joint:
// three point rows on the world axes (correction.wgsl:48-66, 93-104), each applied to working
// copies of the bodies, then the summed correction applied once to the stored rows.
__device__ __forceinline__ void joint_project(const DeviceWorld& w, const dyn_step_params& p, uint32_t j) {
    if (w.jruntime[j].broken != 0u) return;
    const uint4 meta = w.jmeta[j];
    DBody fl = load_dbody(w.hot, meta.z), sl = load_dbody(w.hot, meta.w);
    DBody first = dbody_inert(fl) ? dbody_frozen(fl) : fl;
    DBody second = dbody_inert(sl) ? dbody_frozen(sl) : sl;
    const f3 local_a = xyz(w.janchor_a[j]), local_b = xyz(w.janchor_b[j]);
    f3 total_first = s3(0.0f), total_second = s3(0.0f);
    f3 total_first_ang = s3(0.0f), total_second_ang = s3(0.0f);
    for (uint32_t i = 0; i < 3; ++i) {
        const f3 axis = mk3(i == 0 ? 1.0f : 0.0f, i == 1 ? 1.0f : 0.0f, i == 2 ? 1.0f : 0.0f);
        const f3 pa = arm(first, local_a), pb = arm(second, local_b);
        f3 lin_first = s3(0.0f), lin_second = s3(0.0f);
        const float k = first.inverse_mass + second.inverse_mass;
        if (k > 0.0f) {
            const float magnitude = p.relaxation * (dot(pb - pa, axis) - 0.0f) / k;
            lin_first = axis * (magnitude * first.inverse_mass);
            lin_second = axis * (-magnitude * second.inverse_mass);
        }
        shift_body(&first, lin_first, s3(0.0f));
        shift_body(&second, lin_second, s3(0.0f));
        total_first = total_first + lin_first;
        total_first_ang = total_first_ang + s3(0.0f);
        total_second = total_second + lin_second;
        total_second_ang = total_second_ang + s3(0.0f);
    }
    const bool holds = dot(total_first, total_first) > 0.0f || dot(total_first_ang, total_first_ang) > 0.0f ||
                       dot(total_second, total_second) > 0.0f || dot(total_second_ang, total_second_ang) > 0.0f;
    if (!holds) return;
    BodyHot& ha = w.hot[meta.z];
    BodyHot& hb = w.hot[meta.w];
    const float4 pa4 = ha.pos, ra4 = ha.rot, pb4 = hb.pos, rb4 = hb.rot;
    ha.pos = mk4(xyz(pa4) + total_first, pa4.w);
    ha.rot = normalize4(quat_mul(mk4(total_first_ang * 0.5f, 1.0f), ra4));
    hb.pos = mk4(xyz(pb4) + total_second, pb4.w);
    hb.rot = normalize4(quat_mul(mk4(total_second_ang * 0.5f, 1.0f), rb4));
    const float4 qa = w.resolution[meta.z];
    w.resolution[meta.z] = make_float4(qa.x + total_first.x, qa.y + total_first.y, qa.z + total_first.z, 0.0f);
    const float4 qb = w.resolution[meta.w];
    w.resolution[meta.w] = make_float4(qb.x + total_second.x, qb.y + total_second.y, qb.z + total_second.z, 0.0f);
}

// One warp per group of components (joint_velocity.wgsl:24-54 with a warp for a workgroup).
template <int kPass>
__global__ void __launch_bounds__(32) k_joints(DeviceWorld w, dyn_step_params p) {
    const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (group >= w.jgroup_count) return;  // warp-uniform
    const uint32_t lane = threadIdx.x & 31u;
    const uint4 g = w.jgroups[group];
    const uint32_t lanes = g.z, slot = lane / lanes, li = lane % lanes;
    uint32_t layer_offset = 0, layer_count = 0;
    if (slot < g.y) {
        const uint2 c = w.jcomps[g.x + slot];
        layer_offset = c.x;
        layer_count = c.y;
    }
    const bool residual = kPass == JP_SOLVE && w.ctl[CTL_ROUNDS] == p.solve_iterations;
    for (uint32_t sweep = 0; sweep < 2u; ++sweep) {
        for (uint32_t step = 0; step < g.w; ++step) {
            if (layer_count > step) {
                const uint32_t layer = sweep == 0u ? layer_offset + step : layer_offset + layer_count - 1u - step;
                const uint2 range = w.jlayers[layer];
                for (uint32_t index = li; index < range.y; index += lanes) {
                    const uint32_t j = w.jrows[range.x + index];
                    if (kPass == JP_WARM) {
                        joint_warm(w, j);
                    } else if (kPass == JP_SOLVE) {
                        joint_solve(w, p, j, residual);
                    } else {
                        joint_project(w, p, j);
                    }
                }
            }
            __syncwarp();
        }
    }
}

// COUNTER_JOINTS: the jointed pairs the narrowphase filters this step (joint_filter.wgsl:9-24).
__global__ void k_joint_count(DeviceWorld w) {
    GRID_STRIDE(i, w.jfilter_count) {
        if (w.jruntime[w.jfilter_joint[i]].broken == 0u) add_counter(&w.counters[DYN_COUNTER_JOINTS], 1u);
    }
}

// island_link_constraints.wgsl: every unbroken joint couples its two rows.
__global__ void k_island_link_joints(DeviceWorld w) {
    GRID_STRIDE(j, w.jcount) {
        if (w.jruntime[j].broken != 0u) continue;
        const uint4 meta = w.jmeta[j];
        if (!island_couple(w, meta.z, meta.w)) add_counter(&w.counters[DYN_COUNTER_ISLAND_FAULTS], 1u);
    }
}

}  // namespace dyn
