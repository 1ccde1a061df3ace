//! Raw bindings to libdynamis_cuda.so: the Dynamis rigid-body step (World::step and its
//! differentiation, World::step_backward) re-built as sm_100a CUDA kernels behind the C ABI of
//! include/dynamis_cuda.h. The records are dynamis-abi's own #[repr(C)] records (the library's
//! include/dynamis_abi.h holds the same byte layouts), so nothing is converted at the boundary.
//! Every function returns a DynStatus (0 = DYN_OK); dyn_last_error explains a refusal.
#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_void};

pub use dynamis_abi::{
    BodyDescriptorRecord, BodyEditRecord, BodyStateRecord, ColliderRecord, ConstraintDescriptorRecord,
    ConstraintRuntimeRecord, ContactRecord, QueryHitRecord, QueryRecord, StepParamsRecord,
};

/// An opaque world snapshot (dyn_snapshot).
#[repr(C)]
pub struct DynSnapshot {
    _private: [u8; 0],
}

/// An opaque world handle (dyn_world).
#[repr(C)]
pub struct DynWorld {
    _private: [u8; 0],
}
pub type DynStatus = i32;

/// PhysicsConfig's fields (dyn_config).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct DynConfig {
    pub gravity: [f32; 3],
    pub damping: f32,
    pub angular_damping: f32,
    pub substeps: u32,
    pub solve_iterations: u32,
    pub position_iterations: u32,
    pub relaxation: f32,
    pub slop: f32,
    pub contact_margin: f32,
    pub restitution_threshold: f32,
    pub max_velocity: f32,
    pub max_angular_velocity: f32,
    pub sleep_velocity: f32,
    pub sleep_angular_velocity: f32,
    pub sleep_time: f32,
    pub friction_combine: u32,
    pub restitution_combine: u32,
}

/// Stream capacities (dyn_capacity); zero sizes from the scene.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct DynCapacity {
    pub bodies: u32,
    pub colliders: u32,
    pub pairs: u32,
    pub contacts: u32,
}

/// ColliderDesc, field for field (dyn_collider_desc).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct DynColliderDesc {
    pub shape: u32,
    pub radius: f32,
    pub half_height: f32,
    pub half_extents: [f32; 3],
    pub source: u32,
    pub offset: [f32; 3],
    pub rotation: [f32; 4],
    pub scale: [f32; 3],
    pub friction: f32,
    pub restitution: f32,
    pub rolling_friction: f32,
    pub spin_friction: f32,
    pub contact_frequency: f32,
    pub contact_damping_ratio: f32,
    pub sensor: u32,
    pub events: u32,
    pub collision_group: u32,
    pub collision_mask: u32,
    pub impact_force: f32,
}

/// BodyDesc, field for field (dyn_body_desc); a body owns colliders
/// [collider_first, collider_first + collider_count) of the array passed beside it.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct DynBodyDesc {
    pub position: [f32; 3],
    pub orientation: [f32; 4],
    pub velocity: [f32; 3],
    pub angular_velocity: [f32; 3],
    pub mass: f32,
    pub density: f32,
    pub gravity_scale: f32,
    pub linear_damping: f32,
    pub angular_damping: f32,
    pub sleep_velocity: f32,
    pub sleep_angular_velocity: f32,
    pub collision_group: u32,
    pub collision_mask: u32,
    pub kinematic: u32,
    pub ccd: u32,
    pub collider_first: u32,
    pub collider_count: u32,
}

/// d loss / d one body row's state (dyn_body_grad, 64 bytes).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct DynBodyGrad {
    pub position: [f32; 3],
    pub _pad0: f32,
    pub orientation: [f32; 4],
    pub velocity: [f32; 3],
    pub _pad1: f32,
    pub angular_velocity: [f32; 3],
    pub _pad2: f32,
}

/// A hull shape source as the device holds it (dyn_shape_source_record, records.wgsl's ShapeSource).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct DynShapeSource {
    pub kind: u32,
    pub vertex_offset: u32,
    pub vertex_count: u32,
    pub triangle_offset: u32,
    pub node_offset: u32,
    pub node_count: u32,
    pub cell_offset: u32,
    pub cell_count: u32,
    pub grid_rows: u32,
    pub grid_cols: u32,
    pub _pad0: u32,
    pub _pad1: u32,
    pub local_min: [f32; 3],
    pub _pad2: f32,
    pub local_max: [f32; 3],
    pub _pad3: f32,
}

/// A swept AABB (dyn_aabb_record, records.wgsl's Aabb).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct DynAabb {
    pub min: [f32; 3],
    pub _pad0: f32,
    pub max: [f32; 3],
    pub _pad1: f32,
}

/// The body rows a constraint joins (dyn_constraint_rows_record).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct DynConstraintRows {
    pub first_row: u32,
    pub second_row: u32,
}

/// Launch shapes of the step's kernels (dyn_launch_config); dyn_autotune picks them.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct DynLaunchConfig {
    pub grid_blocks_per_sm: u32,
    pub solve_threads: u32,
    pub gjk_blocks_per_sm: u32,
    pub epa_blocks_per_sm: u32,
}

pub const DYN_OK: DynStatus = 0;
pub const DYN_SOLVER_GUARD_ROW_MASS: u32 = 1;

#[link(name = "dynamis_cuda")]
extern "C" {
    pub fn dyn_abi_version() -> u32;
    pub fn dyn_status_string(status: DynStatus) -> *const c_char;
    pub fn dyn_config_default(out: *mut DynConfig);
    pub fn dyn_collider_desc_default(out: *mut DynColliderDesc);
    pub fn dyn_body_desc_default(out: *mut DynBodyDesc);
    pub fn dyn_world_create(config: *const DynConfig, capacity: *const DynCapacity, device: i32, out: *mut *mut DynWorld) -> DynStatus;
    pub fn dyn_world_destroy(world: *mut DynWorld) -> DynStatus;
    pub fn dyn_last_error(world: *const DynWorld) -> *const c_char;
    pub fn dyn_world_set_stream(world: *mut DynWorld, cuda_stream: *mut c_void) -> DynStatus;
    pub fn dyn_add_hull_from_mesh(world: *mut DynWorld, xyz: *const f32, nv: u32, triangles: *const u32, nt: u32, out_source: *mut u32) -> DynStatus;
    pub fn dyn_add_hull(world: *mut DynWorld, xyz: *const f32, n: u32, out_source: *mut u32) -> DynStatus;
    pub fn dyn_add_hull_mesh(world: *mut DynWorld, xyz: *const f32, nv: u32, triangles: *const u32, nt: u32, out_source: *mut u32) -> DynStatus;
    pub fn dyn_hull_info(world: *const DynWorld, source: u32, vertex_count: *mut u32, triangle_count: *mut u32, volume: *mut f32, centroid: *mut f32) -> DynStatus;
    pub fn dyn_spawn_bodies(world: *mut DynWorld, bodies: *const DynBodyDesc, n: u32, colliders: *const DynColliderDesc, k: u32, out_ids: *mut u32) -> DynStatus;
    pub fn dyn_upload_bodies(world: *mut DynWorld, states: *const BodyStateRecord, descs: *const BodyDescriptorRecord, n: u32, colliders: *const ColliderRecord, owners: *const u32, k: u32) -> DynStatus;
    pub fn dyn_upload_states(world: *mut DynWorld, states: *const BodyStateRecord, n: u32) -> DynStatus;
    pub fn dyn_stream_capacity(world: *const DynWorld, pairs: *mut u32, contacts: *mut u32) -> DynStatus;
    pub fn dyn_scene_sizes(world: *const DynWorld, bodies: *mut u32, dynamic_bodies: *mut u32, colliders: *mut u32, sources: *mut u32, vertices: *mut u32) -> DynStatus;
    pub fn dyn_export_scene(world: *const DynWorld, states: *mut BodyStateRecord, descs: *mut BodyDescriptorRecord, colliders: *mut ColliderRecord, owners: *mut u32, sources: *mut DynShapeSource, vertices_xyzw: *mut f32) -> DynStatus;
    pub fn dyn_step_params_for(world: *const DynWorld, dt: f32, out: *mut StepParamsRecord) -> DynStatus;
    pub fn dyn_step(world: *mut DynWorld, dt: f32) -> DynStatus;
    pub fn dyn_sync(world: *mut DynWorld) -> DynStatus;
    pub fn dyn_device_status(world: *mut DynWorld, status: *mut u32) -> DynStatus;
    pub fn dyn_download_states(world: *mut DynWorld, out: *mut BodyStateRecord, n: u32) -> DynStatus;
    pub fn dyn_read_state(world: *mut DynWorld, body_id: u32, out: *mut BodyStateRecord) -> DynStatus;
    pub fn dyn_read_counters(world: *mut DynWorld, out: *mut u32, n: u32) -> DynStatus;
    pub fn dyn_debug_aabbs(world: *mut DynWorld, out: *mut DynAabb, cap: u32, count: *mut u32) -> DynStatus;
    pub fn dyn_debug_entries(world: *mut DynWorld, keys: *mut u32, infos: *mut u32, cap: u32, count: *mut u32) -> DynStatus;
    pub fn dyn_debug_pairs(world: *mut DynWorld, major: *mut u32, minor: *mut u32, cap: u32, count: *mut u32) -> DynStatus;
    pub fn dyn_debug_contacts(world: *mut DynWorld, out: *mut ContactRecord, cap: u32, count: *mut u32) -> DynStatus;
    pub fn dyn_debug_islands(world: *mut DynWorld, out: *mut u32, cap: u32, count: *mut u32) -> DynStatus;
    pub fn dyn_debug_resting(world: *mut DynWorld, out: *mut u32, cap: u32, count: *mut u32) -> DynStatus;
    pub fn dyn_query(world: *mut DynWorld, queries: *mut QueryRecord, n: u32, hits: *mut QueryHitRecord, hit_capacity: u32) -> DynStatus;
    pub fn dyn_hull_triangles(world: *const DynWorld, source: u32, out: *mut u32, cap: u32, count: *mut u32) -> DynStatus;
    pub fn dyn_set_timing(world: *mut DynWorld, enabled: i32) -> DynStatus;
    pub fn dyn_step_kernel_count(world: *const DynWorld) -> u32;
    pub fn dyn_stage_count() -> u32;
    pub fn dyn_stage_name(stage: u32) -> *const c_char;
    pub fn dyn_stage_timings(world: *mut DynWorld, ms: *mut f32, n: u32) -> DynStatus;
    pub fn dyn_radix_sort(world: *mut DynWorld, major: *mut u32, minor: *mut u32, payload: *mut u32, n: u32, major_digits: u32, minor_digits: u32) -> DynStatus;
    pub fn dyn_observe_bodies(world: *mut DynWorld, body_ids: *const u32, n: u32) -> DynStatus;
    pub fn dyn_stop_observing(world: *mut DynWorld) -> DynStatus;
    pub fn dyn_poll(world: *mut DynWorld) -> DynStatus;
    pub fn dyn_try_state(world: *mut DynWorld, body_id: u32, out: *mut BodyStateRecord, step: *mut u64) -> DynStatus;
    pub fn dyn_try_counters(world: *mut DynWorld, out: *mut u32, n: u32, step: *mut u64) -> DynStatus;
    pub fn dyn_remove_bodies(world: *mut DynWorld, body_ids: *const u32, n: u32) -> DynStatus;
    pub fn dyn_edit_bodies(world: *mut DynWorld, body_ids: *const u32, edits: *const BodyEditRecord, n: u32) -> DynStatus;
    pub fn dyn_set_body_worlds(world: *mut DynWorld, world_of_body: *const u32, n: u32) -> DynStatus;
    pub fn dyn_export_body_worlds(world: *const DynWorld, rows_out: *mut u32) -> DynStatus;
    pub fn dyn_add_ball_joint(world: *mut DynWorld, first_body: u32, second_body: u32, anchor_a: *const f32, anchor_b: *const f32, out_id: *mut u32) -> DynStatus;
    pub fn dyn_add_constraints(world: *mut DynWorld, records: *const ConstraintDescriptorRecord, m: u32, out_first_id: *mut u32) -> DynStatus;
    pub fn dyn_constraint_count(world: *const DynWorld, count: *mut u32) -> DynStatus;
    pub fn dyn_read_constraints(world: *mut DynWorld, out: *mut ConstraintRuntimeRecord, m: u32) -> DynStatus;
    pub fn dyn_export_constraints(world: *const DynWorld, descs: *mut ConstraintDescriptorRecord, rows: *mut DynConstraintRows, runtime: *mut ConstraintRuntimeRecord) -> DynStatus;
    pub fn dyn_joint_plan(world: *const DynWorld, rows: *mut u32, layers: *mut u32, components: *mut u32, layer_count: *mut u32, component_count: *mut u32) -> DynStatus;
    pub fn dyn_radix_sort_static(major: *mut u32, minor: *mut u32, payload: *mut u32, n: u32, major_digits: u32, minor_digits: u32, cuda_stream: *mut c_void) -> DynStatus;
    pub fn dyn_radix_sort_static_status(cuda_stream: *mut c_void, out: *mut u32) -> DynStatus;
    pub fn dyn_set_launch_config(world: *mut DynWorld, config: *const DynLaunchConfig) -> DynStatus;
    pub fn dyn_get_launch_config(world: *const DynWorld, out: *mut DynLaunchConfig) -> DynStatus;
    pub fn dyn_autotune(world: *mut DynWorld, dt: f32, steps: u32, best: *mut DynLaunchConfig, best_ms: *mut f32) -> DynStatus;
    pub fn dyn_snapshot_take(world: *mut DynWorld, out: *mut *mut DynSnapshot) -> DynStatus;
    pub fn dyn_snapshot_restore(world: *mut DynWorld, snapshot: *const DynSnapshot) -> DynStatus;
    pub fn dyn_snapshot_free(snapshot: *mut DynSnapshot) -> DynStatus;
    pub fn dyn_set_solver_guard(world: *mut DynWorld, flags: u32) -> DynStatus;
    pub fn dyn_set_ccd(world: *mut DynWorld, body_id: u32, enabled: i32) -> DynStatus;
    pub fn dyn_clear_device_status(world: *mut DynWorld) -> DynStatus;
    pub fn dyn_debug_sort_fault(world: *mut DynWorld, skipped_tiles: u32, spin_limit: u32) -> DynStatus;
    pub fn dyn_tape_begin(world: *mut DynWorld, checkpoint_interval: u32) -> DynStatus;
    pub fn dyn_tape_end(world: *mut DynWorld) -> DynStatus;
    pub fn dyn_tape_steps(world: *const DynWorld, recorded: *mut u32, reversed: *mut u32) -> DynStatus;
    pub fn dyn_step_backward(world: *mut DynWorld, grad_in: *const DynBodyGrad, grad_out: *mut DynBodyGrad, n: u32) -> DynStatus;
    pub fn dyn_backward(world: *mut DynWorld, grad_in: *const DynBodyGrad, grad_out: *mut DynBodyGrad, n: u32, steps: u32) -> DynStatus;
    pub fn dyn_param_grads(world: *mut DynWorld, inverse_mass: *mut f32, inertia_scale: *mut f32, n: u32, friction: *mut f32, k: u32) -> DynStatus;
    pub fn dyn_set_mass_properties(world: *mut DynWorld, inverse_mass: *const f32, inverse_inertia: *const f32, n: u32) -> DynStatus;
    pub fn dyn_set_friction(world: *mut DynWorld, friction: *const f32, k: u32) -> DynStatus;
}

#[cfg(test)]
mod layout {
    use super::*;
    #[test]
    fn c_abi_sizes() {
        assert_eq!(std::mem::size_of::<DynBodyGrad>(), 64);
        assert_eq!(std::mem::size_of::<DynAabb>(), 32);
        assert_eq!(std::mem::size_of::<DynShapeSource>(), 80);
        assert_eq!(std::mem::size_of::<BodyStateRecord>(), 144);
        assert_eq!(std::mem::size_of::<ContactRecord>(), 352);
    }
}
