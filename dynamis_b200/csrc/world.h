// world.h - host-side state of one world (private to libdynamis_cuda.so).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "dynamis_cuda.h"

namespace dyn {

struct HullSource {
    std::vector<float> vertices;     // xyz triples, in dynamis-hull's order (first appearance over faces)
    std::vector<uint32_t> triangles; // outward triangles over `vertices`
    float volume = 0.0f;
    float centroid[3] = {0.0f, 0.0f, 0.0f};
    float unit_second_moment[6] = {0, 0, 0, 0, 0, 0};
};

// The joint solve order of schedule.rs:105-296 over body rows: `rows` lists joint indices layer by
// layer, `layers` holds (first entry of `rows`, count) pairs, `components` holds (first layer,
// layer count) pairs in the planner's component order, and `groups` packs components into 32-lane
// warps for the device: (first component, component count, lanes per component, deepest stack).
struct JointPlan {
    std::vector<uint32_t> rows;
    std::vector<uint32_t> layers;
    std::vector<uint32_t> components;
    std::vector<uint32_t> groups;
};
void plan_joints(const std::vector<uint32_t>& first, const std::vector<uint32_t>& second, uint32_t body_rows,
                 uint32_t dynamic_count, JointPlan* plan);

struct DeviceState;  // defined in world.cu

// The observation ring (observation.rs, dynamis-gpu/src/readback.rs:158-173): after each step the
// observed bodies' state records and the counters are copied on the world's stream into one of a
// few pinned host slots; reads take the newest slot whose copy has completed and never wait.
constexpr uint32_t kObservationSlots = 4;
struct ObservationSlot {
    void* states = nullptr;    // pinned dyn_body_state_record[capacity]
    void* counters = nullptr;  // pinned uint32_t[64]
    uint32_t capacity = 0;
    uint32_t count = 0;        // records copied
    void* done = nullptr;      // cudaEvent_t recorded after the copies
    std::vector<uint32_t> index_of_id;  // body id -> record, built from the records on the first read
    uint64_t step = 0;
    bool pending = false, ready = false;
};
struct Observer {
    bool active = false, all = false;
    std::vector<uint32_t> ids;  // the observed bodies (when not all)
    ObservationSlot slots[kObservationSlots];
    int latest = -1;            // newest completed slot
    void* ids_dev = nullptr;    // device copy of ids, resolved to rows on the device at each copy
    uint32_t ids_dev_capacity = 0;
    bool ids_dirty = false;     // ids changed since the device copy was made
    uint64_t superseded = 0;    // copies replaced by a newer one before they completed
};

}  // namespace dyn

struct dyn_world {
    dyn_config config{};
    dyn_capacity capacity{};
    int32_t device = 0;
    std::string last_error;
    // shape pool
    std::vector<dyn::HullSource> hulls;
    // scene in spawn order (body id = spawn index)
    std::vector<dyn_body_state_record> spawn_states;
    std::vector<dyn_body_descriptor_record> spawn_descs;
    std::vector<dyn_collider_record> spawn_colliders;
    std::vector<uint32_t> spawn_owner;  // body id of each collider
    std::vector<uint8_t> removed;       // by body id: removed from the world (ids are not reused)
    // scene as rows (dynamic rows first), rebuilt when the scene changes
    bool rows_dirty = true;
    bool raw_rows = false;  // scene came from dyn_upload_bodies
    std::vector<dyn_body_state_record> states;
    std::vector<dyn_body_descriptor_record> descs;
    std::vector<dyn_collider_record> colliders;
    std::vector<uint32_t> owners;
    std::vector<uint32_t> row_of_id;
    uint32_t dynamic_count = 0;
    // batched worlds: the sub-world of every body by id (empty: one world) and of every row
    std::vector<uint32_t> world_of_id;
    std::vector<uint32_t> body_world;
    // constraints in creation order (constraint id = index); rows and plan derived with the rows
    std::vector<dyn_constraint_descriptor_record> joint_descs;
    std::vector<dyn_constraint_runtime_record> joint_runtime;  // initial runtime records
    std::vector<dyn_constraint_rows_record> joint_rows;
    dyn::JointPlan joint_plan;
    bool joints_dirty = false;  // the device's joint buffers and plan are out of date
    bool scene_dirty = false;   // the device's scene is out of date although the rows are current
    // body commands queued for the next step (body id, edit), in the order given
    std::vector<uint32_t> edit_ids;
    std::vector<dyn_body_edit_record> edits;
    bool timing = false;
    uint32_t solver_guard = 0;  // DYN_SOLVER_GUARD_* bits (dyn_set_solver_guard)
    dyn_launch_config launch{16u, 128u, 6u, 8u};  // applied when the device state is made
    void* user_stream = nullptr;  // caller's cudaStream_t (dyn_world_set_stream)
    uint64_t steps_taken = 0;     // dyn_step calls since creation
    dyn::Observer observer;
    dyn::DeviceState* dev = nullptr;
};

namespace dyn {
dyn_status fail(dyn_world* w, dyn_status status, const std::string& what);
void rebuild_rows(dyn_world* w);
dyn_status rebuild_joints(dyn_world* w);
// Copies the device's current body states into the spawn-order store (a no-op before the first step).
dyn_status sync_spawn_states(dyn_world* w);
std::vector<dyn_shape_source_record> shape_sources(const dyn_world* w, std::vector<float>* vertices_xyzw);
void destroy_device(dyn_world* w);
// Arms the next dyn_radix_sort_static call with a fault (static_sort.cu; dyn_debug_sort_fault).
dyn_status static_sort_fault(uint32_t skipped_tiles, uint32_t spin_limit);
}  // namespace dyn
