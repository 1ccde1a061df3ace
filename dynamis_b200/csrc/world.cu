// world.cu - device side of the C ABI: HBM allocation, record conversion, the step as a CUDA
// graph, readback and the parity hooks.
//
// The step replays one captured graph per (dt, archive parity): the current and archived contact
// sets swap roles every step (contact_archive.wgsl copies instead), so two graphs alternate.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "adjoint.cuh"
#include "ccd.cuh"
#include "joints.cuh"
#include "query.cuh"
#include "rest.cuh"
#include "step.cuh"
#include "world.h"

namespace dyn {

enum Stage : uint32_t {
    ST_BEGIN = 0,
    ST_AABB,
    ST_ENTRIES,
    ST_ENTRY_SORT,
    ST_PAIRS,
    ST_NARROWPHASE,
    ST_COMPACT,
    ST_IDENTITY,
    ST_ISLANDS,
    ST_WAKE_LIVE,
    ST_SOLVER_PREPARE,
    ST_INTEGRATE,
    ST_WARM,
    ST_VELOCITY,
    ST_ADVANCE,
    ST_POSITION,
    ST_CCD,
    ST_SLEEP,
    ST_COUNT
};
static const char* kStageNames[ST_COUNT] = {"begin",       "aabb",     "entries",   "entry_sort",     "pairs",
                                            "narrowphase", "compact",  "identity",       "islands",
                                            "wake_live",   "solver_prepare", "integrate", "warm_start", "velocity",
                                            "advance",     "position", "ccd",       "sleep"};

// A recorded trajectory for the adjoint (dyn_tape_begin ... dyn_tape_end): checkpoints on the
// device, the taped segment and the gradient buffers.
struct Checkpoint {
    void* base = nullptr;  // one device block holding the parts save_checkpoint lists, 256-byte aligned
    size_t bytes = 0;
    uint32_t parity = 0;
};
struct TapeHost {
    bool active = false;
    uint32_t interval = 10;
    uint32_t recorded = 0;  // steps recorded since dyn_tape_begin
    uint32_t reversed = 0;  // of those, the last ones already reversed
    float dt = 0.0f;        // every recorded step's timestep
    // checkpoint j: the world before recorded step j * interval. The blocks, the tape, the gradient
    // buffers and the graphs stay allocated from one tape to the next (a tape of the same shape
    // allocates nothing) until the device state goes.
    std::vector<Checkpoint> checkpoints;
    uint32_t checkpoint_count = 0;  // of those, the current tape's
    Checkpoint end;                 // the world after the last recorded step (kept from the first backward on)
    bool have_end = false;
    std::vector<std::vector<uint32_t>> edit_ids;  // each recorded step's queued edits, replayed with it
    std::vector<std::vector<dyn_body_edit_record>> edits;
    int32_t segment = -1;  // the segment whose steps the tape slots hold
    TapeView view{};
    std::vector<void*> tape_allocs;
    AdjView adj{};
    std::vector<void*> adj_allocs;
    dyn_body_grad* grad_staging = nullptr;  // [n_cap] ABI gradient records
    uint32_t* patch_rows = nullptr;         // [n_cap] rows and masks of a step's PATCH edits
    uint32_t* patch_masks = nullptr;
    cudaGraphExec_t taped[2] = {nullptr, nullptr};
    cudaGraphExec_t back = nullptr;
};

struct DeviceState {
    cudaStream_t own_stream = nullptr;
    // a second stream the captured step forks onto for kernels independent of the main line
    cudaStream_t side_stream = nullptr;
    cudaStream_t side_stream2 = nullptr;
    cudaEvent_t fork_events[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t join_events[4] = {nullptr, nullptr, nullptr, nullptr};
    // the last kStepsInFlight steps' completion events: dyn_step waits for the oldest before it
    // queues another, so what the device reports (the pair demand) is at most that many steps old
    cudaEvent_t inflight[4] = {nullptr, nullptr, nullptr, nullptr};
    bool inflight_used[4] = {false, false, false, false};
    uint32_t inflight_next = 0;
    cudaStream_t stream = nullptr;
    DeviceWorld dw{};
    std::vector<void*> allocs;
    uint32_t* spill_host = nullptr;  // host-mapped mailbox of stream demand (DeviceWorld::spill)
    uint32_t n_cap = 0, k_cap = 0, e_cap = 0, p_cap = 0, c_cap = 0;
    uint32_t id_cap = 0;  // body ids the row_of_id table holds (ids of removed bodies are not reused)
    uint32_t src_cap = 0, vert_cap = 0, tri_cap = 0;
    dyn_shape_source_record* sources = nullptr;
    float4* vertices = nullptr;
    uint4* hull_tris = nullptr;       // the hulls' triangles (scene queries)
    uint2* hull_tri_range = nullptr;  // [source]: first triangle, count
    // a query batch's records and hits on the device (dyn_query), grown as batches need
    dyn_query_record* query_buf = nullptr;
    dyn_query_hit_record* hit_buf = nullptr;
    // a query's own grid: its entries and its counters and control words, so that a query between
    // steps leaves the step's kept grid runs and counters as they were
    float4* query_entries = nullptr;
    uint32_t* query_words = nullptr;
    uint32_t query_cap = 0, hit_cap = 0;
    // sort and scan scratch
    uint32_t* hist = nullptr;          // 8 x 256
    uint32_t* tile_counters = nullptr; // 16
    uint32_t* lookback = nullptr;
    size_t lookback_words = 0;
    uint32_t* sort_alt0 = nullptr;  // operator scratch (dyn_radix_sort)
    uint32_t* sort_alt1 = nullptr;
    uint32_t* sort_alt2 = nullptr;
    uint32_t sort_alt_cap = 0;
    // test hook (dyn_debug_sort_fault): the next dyn_radix_sort starts each digit pass's tile
    // ticket at sort_fault_skip (tiles below it never run) and polls at most sort_fault_limit times
    bool sort_fault_armed = false;
    uint32_t sort_fault_skip = 0;
    uint32_t sort_fault_limit = kLookbackSpinLimit;
    dyn_body_state_record* staging = nullptr;  // n_cap ABI state records
    // the two frozen-contact stores (rest.cuh); a step reads rest_*[parity] and writes the other
    uint4* rest_ids[2] = {nullptr, nullptr};
    uint2* rest_slots[2] = {nullptr, nullptr};
    uint32_t rest_cap = 0;
    std::vector<void*> joint_allocs;  // constraint buffers, rebuilt whenever the constraint set changes
    // body edits: once a world has taken edits its step graph runs k_clear_inputs, k_body_edits and
    // k_begin<false>; before that, k_begin<true> alone
    bool edit_graphs = false;
    bool edits_pending_on_device = false;  // *edit_count is non-zero
    dyn_body_edit_record* edit_buffer = nullptr;
    uint4* edit_run_buffer = nullptr;
    uint32_t edit_capacity = 0;
    // graphs
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    float graph_dt = -1.0f;
    uint32_t parity = 0;  // which contact set is current for the next step
    uint32_t last_parity = 0;
    bool stepped = false;
    bool uploaded = false;  // the current scene's records are on the device
    uint32_t graph_kernels = 0;  // kernel nodes in one step's graph
    uint64_t scene_epoch = 0;    // scene uploads so far (a snapshot belongs to one scene)
    uint32_t sms = 148;          // multiprocessors of the device (read when the device state is made)
    dyn_launch_config launch{16u, 128u, 6u, 8u};  // dyn_set_launch_config / dyn_autotune
    bool tuning = false;         // dyn_autotune is running trials: the contact stream keeps its layout
    dyn_step_params params{};
    // timing
    std::vector<cudaEvent_t> events;
    std::vector<uint32_t> event_stage;
    float stage_ms[ST_COUNT] = {0};
    TapeHost tape;
};
// Frees every buffer and graph of the differentiation (destroy_device; defined with the tape code).
void free_tape_memory(DeviceState* d);

namespace {

#define DYN_CUDA(call)                                                                                  \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return fail(w, DYN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
dyn_status alloc(dyn_world* w, DeviceState* d, T** out, size_t count) {
    void* p = nullptr;
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    DYN_CUDA(cudaMalloc(&p, bytes));
    DYN_CUDA(cudaMemsetAsync(p, 0, bytes, d->stream));
    d->allocs.push_back(p);
    *out = static_cast<T*>(p);
    return DYN_OK;
}

dyn_status alloc_contacts(dyn_world* w, DeviceState* d, ContactSet* s, uint32_t cap) {
    dyn_status st;
    if ((st = alloc(w, d, &s->normal, cap))) return st;
    if ((st = alloc(w, d, &s->rows, cap))) return st;
    if ((st = alloc(w, d, &s->mat, cap))) return st;
    if ((st = alloc(w, d, &s->ids, cap))) return st;
    if ((st = alloc(w, d, &s->ids2, cap))) return st;
    if ((st = alloc(w, d, &s->extra, cap))) return st;
    if ((st = alloc(w, d, &s->la, (size_t)4 * cap))) return st;
    if ((st = alloc(w, d, &s->lb, (size_t)4 * cap))) return st;
    if ((st = alloc(w, d, &s->acc, (size_t)4 * cap))) return st;
    if ((st = alloc(w, d, &s->pos, (size_t)4 * cap))) return st;
    return DYN_OK;
}

uint32_t key_words(uint32_t n) {
    uint32_t m = n > 0 ? n - 1 : 0;
    uint32_t bits = m == 0 ? 0 : 32 - (uint32_t)__builtin_clz(m);
    uint32_t words = (bits + 7) / 8;
    return words < 1 ? 1 : (words > 4 ? 4 : words);
}
inline uint32_t div_up(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }
// Grid-stride launches: enough blocks for n threads, at most 16 blocks per SM of the device.
inline uint32_t blocks_for(const DeviceState* d, uint32_t n, uint32_t threads) {
    uint32_t b = div_up(std::max<uint32_t>(n, 1), threads);
    return std::min<uint32_t>(b, d->sms * d->launch.grid_blocks_per_sm);
}

void release_graphs(DeviceState* d) {
    for (auto& e : d->exec) {
        if (e) cudaGraphExecDestroy(e);
        e = nullptr;
    }
    for (auto& e : d->tape.taped) {
        if (e) cudaGraphExecDestroy(e);
        e = nullptr;
    }
    if (d->tape.back) cudaGraphExecDestroy(d->tape.back);
    d->tape.back = nullptr;
    d->graph_dt = -1.0f;
}

// Allocates HBM for the current scene (capacities are the larger of declared and needed).
dyn_status ensure_device(dyn_world* w) {
    rebuild_rows(w);
    uint32_t n = (uint32_t)w->states.size();
    uint32_t k = (uint32_t)w->colliders.size();
    std::vector<float> verts;
    std::vector<dyn_shape_source_record> srcs = shape_sources(w, &verts);
    uint32_t ns = (uint32_t)srcs.size(), nv = (uint32_t)(verts.size() / 4);
    uint32_t nt = 0;
    for (const HullSource& h : w->hulls) nt += (uint32_t)(h.triangles.size() / 3);
    const uint32_t ids = (uint32_t)w->row_of_id.size();
    DeviceState* d = w->dev;
    bool fits = d && n <= d->n_cap && k <= d->k_cap && ns <= d->src_cap && nv <= d->vert_cap && nt <= d->tri_cap &&
                ids <= d->id_cap;
    if (!fits) {
        if (d) destroy_device(w);
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return fail(w, DYN_ERR_NO_DEVICE, "no CUDA device");
        if (w->device < 0 || w->device >= count) return fail(w, DYN_ERR_NO_DEVICE, "CUDA device ordinal out of range");
        DYN_CUDA(cudaSetDevice(w->device));
        // the GJK/EPA frames of the narrowphase live in per-thread local memory
        DYN_CUDA(cudaDeviceSetLimit(cudaLimitStackSize, 16384));
        d = new DeviceState();
        w->dev = d;
        int sm_count = 0;
        DYN_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, w->device));
        d->sms = (uint32_t)std::max(sm_count, 1);
        d->launch = w->launch;
        DYN_CUDA(cudaStreamCreateWithFlags(&d->own_stream, cudaStreamNonBlocking));
        DYN_CUDA(cudaStreamCreateWithFlags(&d->side_stream, cudaStreamNonBlocking));
        DYN_CUDA(cudaStreamCreateWithFlags(&d->side_stream2, cudaStreamNonBlocking));
        for (uint32_t i = 0; i < 4; ++i) {
            DYN_CUDA(cudaEventCreateWithFlags(&d->fork_events[i], cudaEventDisableTiming));
            DYN_CUDA(cudaEventCreateWithFlags(&d->join_events[i], cudaEventDisableTiming));
            DYN_CUDA(cudaEventCreateWithFlags(&d->inflight[i], cudaEventDisableTiming));
        }
        d->stream = w->user_stream ? static_cast<cudaStream_t>(w->user_stream) : d->own_stream;
        DYN_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&d->spill_host), 4 * sizeof(uint32_t), cudaHostAllocMapped));
        std::memset(d->spill_host, 0, 4 * sizeof(uint32_t));
        DYN_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&d->dw.spill), d->spill_host, 0));
        d->n_cap = std::max(n, w->capacity.bodies);
        d->k_cap = std::max(k, w->capacity.colliders);
        d->e_cap = 8u * std::max(d->k_cap, 1u);
        d->p_cap = w->capacity.pairs ? w->capacity.pairs : 16u * std::max(d->k_cap, 64u);
        d->c_cap = w->capacity.contacts ? w->capacity.contacts : 16u * std::max(d->k_cap, 64u);
        d->src_cap = std::max(ns, 1u);
        d->vert_cap = std::max(nv, 1u);
        d->tri_cap = std::max(nt, 1u);
        DeviceWorld& dw = d->dw;
        dyn_status st;
#define A(ptr, count) if ((st = alloc(w, d, &(ptr), (count)))) return st
        uint32_t N = d->n_cap, K = d->k_cap, E = d->e_cap, P = d->p_cap, C = d->c_cap;
        A(dw.hot, N);
        A(dw.prev_pos, N);
        A(dw.prev_rot, N);
        A(dw.force, N);
        A(dw.torque, N);
        A(dw.ident, N);
        A(dw.sleep_timer, N);
        A(dw.damp, N);
        A(dw.thresh, N);
        A(dw.inert0, N);
        A(dw.inert1, N);
        A(dw.activity, N);
        A(dw.motion, N);
        A(dw.wake_flags, N);
        d->id_cap = std::max(N, ids + ids / 2);  // room for spawns after removals
        A(dw.row_of_id, d->id_cap);
        A(dw.body_world, N);
        A(dw.ccd_time, N);
        A(dw.ccd_key, N);
        A(dw.ccd_impact, 2 * (size_t)N);
        A(dw.edit_count, 1);
        A(dw.c_owner, K);
        A(dw.c_kind, K);
        A(dw.c_offset, K);
        A(dw.c_lrot, K);
        A(dw.c_half, K);
        A(dw.c_mat, K);
        A(dw.c_mat2, K);
        A(dw.c_filter, K);
        A(dw.c_scale, K);
        A(d->sources, d->src_cap);
        A(d->vertices, d->vert_cap);
        A(d->hull_tris, d->tri_cap);
        A(d->hull_tri_range, d->src_cap);
        A(dw.aabb, 2 * (size_t)K);
        A(dw.c_class, K);
        A(dw.c_level, K);
        A(dw.entry_count, K);
        A(dw.entry_offset, K);
        A(dw.ekey, E);
        A(dw.eval, E);
        A(dw.ekey_alt, E);
        A(dw.eval_alt, E);
        A(dw.entries, 2 * (size_t)E);
        A(dw.c_run, K);
        A(dw.c_held, K);
        A(dw.run_count, 3 * (size_t)K);
        A(dw.run_offset, 3 * (size_t)K);
        A(dw.run_key, 3 * (size_t)E);
        A(dw.run_val, 3 * (size_t)E);
        A(dw.held, HELD_COUNT);
        A(dw.init_pos, E);
        dw.cell_bits = 10u;
        while (dw.cell_bits < 31u && ((size_t)1 << dw.cell_bits) < 2 * (size_t)E) ++dw.cell_bits;
        A(dw.cell_table, (size_t)1 << dw.cell_bits);
        A(dw.erun, E);
        A(dw.pmaj, P);
        A(dw.pmin, P);
        // the staging set and its sort keys hold every contact the narrowphase finds: one per pair at most
        A(dw.cmaj, P);
        A(dw.cmin, P);
        A(dw.cval, P);
        A(dw.cmaj_alt, P);
        A(dw.cmin_alt, P);
        A(dw.cval_alt, P);
        A(dw.np_list, (PC_COUNT + 1) * (size_t)P);
        A(dw.epa_list, P);
        A(dw.epa_simplex, 4 * (size_t)P);
        A(dw.probe_list, P);
        A(dw.probe_data, 6 * (size_t)P);
        A(dw.hit_list, P);
        A(dw.hit_data, 2 * (size_t)P);
        A(dw.matched, C);
        A(dw.srows.arm_a, 4 * (size_t)C);
        A(dw.srows.arm_b, 4 * (size_t)C);
        A(dw.srows.masses, 4 * (size_t)C);
        A(dw.srows.tangent1, C);
        A(dw.srows.tangent2, C);
        A(dw.parents, N);
        A(dw.istate, N);
        A(dw.live, N);
        A(dw.solver_rows, N);
        A(dw.row_flag, N);
        A(dw.row_offset, N);
        A(dw.vdelta, 8 * (size_t)N);
        A(dw.pdelta, 8 * (size_t)N);
        A(dw.contributions, N);
        A(dw.resolution, N);
        A(dw.pd3, 3 * (size_t)N);
        A(dw.cnt3, 3 * (size_t)N);
        A(dw.resolution_alt, N);
        A(dw.cowner, C);
        // the frozen-contact stores: as many as the contact stream held when the world was made
        d->rest_cap = C;
        for (int r = 0; r < 2; ++r) {
            A(d->rest_ids[r], C);
            A(d->rest_slots[r], C);
        }
        A(dw.counters, 64);
        A(dw.ctl, CTL_COUNT);
        A(d->staging, N);
        A(d->hist, 8 * 256);
        A(d->tile_counters, 16);
        uint32_t max_tiles = std::max(div_up(std::max(E, P), kSortTile), 1u);
        d->lookback_words = (size_t)8 * max_tiles * 256;
        A(d->lookback, d->lookback_words);
#undef A
        if ((st = alloc_contacts(w, d, &dw.tmp, P))) return st;
        dw.s_cap = P;
        if ((st = alloc_contacts(w, d, &dw.cur, C))) return st;
        if ((st = alloc_contacts(w, d, &dw.arc, C))) return st;
        dw.e_cap = E;
        dw.n_cap = N;
        dw.p_cap = P;
        dw.c_cap = C;
        dw.sources = d->sources;
        dw.vertices = d->vertices;
        dw.hull_tris = d->hull_tris;
        dw.hull_tri_range = d->hull_tri_range;
    }
    return DYN_OK;
}

// Converts the host rows to the device layout and uploads them.
// The device's constraint runtime (accumulated impulses, reactions, broken flags) back into the
// host copy, so that re-uploading the scene or the constraint set keeps what the steps built.
dyn_status save_joint_runtime(dyn_world* w) {
    DeviceState* d = w->dev;
    if (!d || !d->stepped || d->dw.jcount == 0) return DYN_OK;
    uint32_t m = std::min<uint32_t>(d->dw.jcount, (uint32_t)w->joint_runtime.size());
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    DYN_CUDA(cudaMemcpy(w->joint_runtime.data(), d->dw.jruntime, (size_t)m * sizeof(dyn_constraint_runtime_record),
                        cudaMemcpyDeviceToHost));
    return DYN_OK;
}

// Constraint descriptors, runtime, solve order and collision filter onto the device.
dyn_status upload_joints(dyn_world* w) {
    dyn_status st = rebuild_joints(w);
    if (st) return st;
    DeviceState* d = w->dev;
    DeviceWorld& dw = d->dw;
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    for (void* p : d->joint_allocs) cudaFree(p);
    d->joint_allocs.clear();
    dw.jcount = dw.jgroup_count = dw.jfilter_count = 0;
    release_graphs(d);
    w->joints_dirty = false;
    d->scene_epoch += 1;  // the constraint set is part of what a snapshot restores
    const uint32_t m = (uint32_t)w->joint_descs.size();
    if (m == 0) return DYN_OK;
    const JointPlan& plan = w->joint_plan;
    std::vector<uint4> meta(m);
    std::vector<float4> anchor_a(m), anchor_b(m);
    struct Filter {
        uint32_t a, b, joint;
    };
    std::vector<Filter> filter;
    for (uint32_t j = 0; j < m; ++j) {
        const dyn_constraint_descriptor_record& c = w->joint_descs[j];
        const dyn_constraint_rows_record& r = w->joint_rows[j];
        meta[j] = make_uint4(c.kind, c.flags, r.first_row, r.second_row);
        anchor_a[j] = make_float4(c.anchor_a[0], c.anchor_a[1], c.anchor_a[2], c.break_force);
        anchor_b[j] = make_float4(c.anchor_b[0], c.anchor_b[1], c.anchor_b[2], c.break_torque);
        if (c.flags & DYN_CONSTRAINT_DISABLE_COLLISIONS)
            filter.push_back(Filter{std::min(r.first_row, r.second_row), std::max(r.first_row, r.second_row), j});
    }
    std::sort(filter.begin(), filter.end(), [](const Filter& x, const Filter& y) {
        return x.a != y.a ? x.a < y.a : (x.b != y.b ? x.b < y.b : x.joint < y.joint);
    });
    std::vector<uint2> fpairs(filter.size());
    std::vector<uint32_t> fjoint(filter.size());
    for (size_t i = 0; i < filter.size(); ++i) {
        fpairs[i] = make_uint2(filter[i].a, filter[i].b);
        fjoint[i] = filter[i].joint;
    }
    auto grab = [&](void** ptr, size_t bytes) -> dyn_status {
        DYN_CUDA(cudaMalloc(ptr, std::max<size_t>(bytes, 16)));
        d->joint_allocs.push_back(*ptr);
        return DYN_OK;
    };
#define JA(field, bytes) if ((st = grab(reinterpret_cast<void**>(&dw.field), (bytes)))) return st
    JA(jmeta, m * sizeof(uint4));
    JA(janchor_a, m * sizeof(float4));
    JA(janchor_b, m * sizeof(float4));
    JA(jruntime, m * sizeof(dyn_constraint_runtime_record));
    JA(jrows, plan.rows.size() * 4);
    JA(jlayers, plan.layers.size() * 4);
    JA(jcomps, plan.components.size() * 4);
    JA(jgroups, plan.groups.size() * 4);
    JA(jfilter, fpairs.size() * sizeof(uint2));
    JA(jfilter_joint, fjoint.size() * 4);
#undef JA
    cudaStream_t s = d->stream;
    DYN_CUDA(cudaMemcpyAsync(dw.jmeta, meta.data(), m * sizeof(uint4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.janchor_a, anchor_a.data(), m * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.janchor_b, anchor_b.data(), m * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.jruntime, w->joint_runtime.data(), m * sizeof(dyn_constraint_runtime_record),
                             cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.jrows, plan.rows.data(), plan.rows.size() * 4, cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.jlayers, plan.layers.data(), plan.layers.size() * 4, cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.jcomps, plan.components.data(), plan.components.size() * 4, cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.jgroups, plan.groups.data(), plan.groups.size() * 4, cudaMemcpyHostToDevice, s));
    if (!fpairs.empty()) {
        DYN_CUDA(cudaMemcpyAsync(dw.jfilter, fpairs.data(), fpairs.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
        DYN_CUDA(cudaMemcpyAsync(dw.jfilter_joint, fjoint.data(), fjoint.size() * 4, cudaMemcpyHostToDevice, s));
    }
    DYN_CUDA(cudaStreamSynchronize(s));
    dw.jcount = m;
    dw.jgroup_count = (uint32_t)(plan.groups.size() / 4);
    dw.jfilter_count = (uint32_t)fpairs.size();
    return DYN_OK;
}

dyn_status upload_scene(dyn_world* w) {
    dyn_status st = ensure_device(w);
    if (st) return st;
    DeviceState* d = w->dev;
    DeviceWorld& dw = d->dw;
    uint32_t n = (uint32_t)w->states.size(), k = (uint32_t)w->colliders.size();
    dw.n = n;
    dw.nd = w->dynamic_count;
    dw.k = k;
    dw.id_count = (uint32_t)w->row_of_id.size();
    std::vector<BodyHot> hot(n);
    std::vector<float4> prev_pos(n), prev_rot(n), force(n), torque(n), damp(n), inert0(n);
    std::vector<uint4> ident(n);
    std::vector<float> timer(n);
    std::vector<float2> thresh(n), inert1(n);
    for (uint32_t i = 0; i < n; ++i) {
        const dyn_body_state_record& s = w->states[i];
        const dyn_body_descriptor_record& c = w->descs[i];
        BodyHot& h = hot[i];
        h.pos = make_float4(s.position[0], s.position[1], s.position[2], c.inverse_mass);
        h.rot = make_float4(s.orientation[0], s.orientation[1], s.orientation[2], s.orientation[3]);
        h.vel = make_float4(s.velocity[0], s.velocity[1], s.velocity[2], 0.0f);
        h.ang = make_float4(s.angular_velocity[0], s.angular_velocity[1], s.angular_velocity[2], 0.0f);
        h.com = make_float4(c.com[0], c.com[1], c.com[2], 0.0f);
        h.ii0 = make_float4(c.inverse_inertia[0], c.inverse_inertia[1], c.inverse_inertia[2], c.inverse_inertia[3]);
        h.ii1 = make_float4(c.inverse_inertia[4], c.inverse_inertia[5], 0.0f, 0.0f);
        h.aux = make_uint4(s.sleeping, c.flags, 0u, 0u);
        prev_pos[i] = make_float4(s.prev_position[0], s.prev_position[1], s.prev_position[2], 0.0f);
        prev_rot[i] = make_float4(s.prev_orientation[0], s.prev_orientation[1], s.prev_orientation[2], s.prev_orientation[3]);
        force[i] = make_float4(s.force[0], s.force[1], s.force[2], 0.0f);
        torque[i] = make_float4(s.torque[0], s.torque[1], s.torque[2], 0.0f);
        ident[i] = make_uint4(s.body_id, s.generation, c.collision_group, c.collision_mask);
        timer[i] = s.sleep_timer;
        damp[i] = make_float4(c.linear_damping, c.angular_damping, c.gravity_scale, 0.0f);
        thresh[i] = make_float2(c.sleep_velocity, c.sleep_angular_velocity);
        inert0[i] = make_float4(c.inertia[0], c.inertia[1], c.inertia[2], c.inertia[3]);
        inert1[i] = make_float2(c.inertia[4], c.inertia[5]);
    }
    std::vector<uint4> ckind(k);
    std::vector<float4> coff(k), clrot(k), chalf(k), cmat(k), cmat2(k), cscale(k);
    std::vector<uint2> cfilter(k);
    for (uint32_t i = 0; i < k; ++i) {
        const dyn_collider_record& c = w->colliders[i];
        ckind[i] = make_uint4(c.kind, c.flags, c.source, 0u);
        coff[i] = make_float4(c.local_offset[0], c.local_offset[1], c.local_offset[2], c.radius);
        clrot[i] = make_float4(c.local_rotation[0], c.local_rotation[1], c.local_rotation[2], c.local_rotation[3]);
        chalf[i] = make_float4(c.half_extents[0], c.half_extents[1], c.half_extents[2], c.half_height);
        cmat[i] = make_float4(c.friction, c.restitution, c.rolling_friction, c.spin_friction);
        cmat2[i] = make_float4(c.relaxation, c.damping_ratio, c.impact_force, 0.0f);
        cfilter[i] = make_uint2(c.collision_group, c.collision_mask);
        cscale[i] = make_float4(c.scale[0], c.scale[1], c.scale[2], 0.0f);
    }
    std::vector<float> verts;
    std::vector<dyn_shape_source_record> srcs = shape_sources(w, &verts);
    cudaStream_t s = d->stream;
    // Host vectors live until the synchronisation at the end of this function.
    DYN_CUDA(cudaMemcpyAsync(dw.hot, hot.data(), n * sizeof(BodyHot), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.prev_pos, prev_pos.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.prev_rot, prev_rot.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.force, force.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.torque, torque.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.ident, ident.data(), n * sizeof(uint4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.sleep_timer, timer.data(), n * sizeof(float), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.damp, damp.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.thresh, thresh.data(), n * sizeof(float2), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.inert0, inert0.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.inert1, inert1.data(), n * sizeof(float2), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.row_of_id, w->row_of_id.data(), w->row_of_id.size() * 4, cudaMemcpyHostToDevice, s));
    std::vector<uint32_t> body_world(n, 0u);
    for (uint32_t i = 0; i < n && i < w->body_world.size(); ++i) body_world[i] = w->body_world[i];
    DYN_CUDA(cudaMemcpyAsync(dw.body_world, body_world.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemsetAsync(dw.wake_flags, 0, (size_t)d->n_cap * 4, s));
    DYN_CUDA(cudaMemcpyAsync(dw.c_owner, w->owners.data(), k * 4, cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.c_kind, ckind.data(), k * sizeof(uint4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.c_offset, coff.data(), k * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.c_lrot, clrot.data(), k * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.c_half, chalf.data(), k * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.c_mat, cmat.data(), k * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.c_mat2, cmat2.data(), k * sizeof(float4), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.c_filter, cfilter.data(), k * sizeof(uint2), cudaMemcpyHostToDevice, s));
    DYN_CUDA(cudaMemcpyAsync(dw.c_scale, cscale.data(), k * sizeof(float4), cudaMemcpyHostToDevice, s));
    std::vector<uint4> tris;
    std::vector<uint2> tri_range(srcs.size());
    for (size_t h = 0; h < w->hulls.size(); ++h) {
        const std::vector<uint32_t>& t = w->hulls[h].triangles;
        tri_range[h] = make_uint2((uint32_t)tris.size(), (uint32_t)(t.size() / 3));
        for (size_t i = 0; i + 2 < t.size(); i += 3) tris.push_back(make_uint4(t[i], t[i + 1], t[i + 2], 0u));
    }
    if (!srcs.empty()) {
        DYN_CUDA(cudaMemcpyAsync(d->sources, srcs.data(), srcs.size() * sizeof(dyn_shape_source_record), cudaMemcpyHostToDevice, s));
        DYN_CUDA(cudaMemcpyAsync(d->vertices, verts.data(), verts.size() * sizeof(float), cudaMemcpyHostToDevice, s));
        DYN_CUDA(cudaMemcpyAsync(d->hull_tri_range, tri_range.data(), tri_range.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
    }
    if (!tris.empty()) {
        DYN_CUDA(cudaMemcpyAsync(d->hull_tris, tris.data(), tris.size() * sizeof(uint4), cudaMemcpyHostToDevice, s));
    }
    // a fresh scene has no archived contacts and no device status; the frozen contacts, kept by
    // body id and generation, carry over (a spawn or a removal does not thaw them), so the store the
    // next step reads moves to the one parity 0 reads
    if (d->parity != 0u && d->rest_cap) {
        DYN_CUDA(cudaMemcpyAsync(d->rest_ids[0], d->rest_ids[1], (size_t)d->rest_cap * sizeof(uint4), cudaMemcpyDeviceToDevice, s));
        DYN_CUDA(cudaMemcpyAsync(d->rest_slots[0], d->rest_slots[1], (size_t)d->rest_cap * sizeof(uint2), cudaMemcpyDeviceToDevice, s));
    }
    DYN_CUDA(cudaMemsetAsync(dw.ctl, 0, CTL_RESTING * 4, s));
    DYN_CUDA(cudaMemsetAsync(dw.ctl + CTL_RESTING + 1, 0, (CTL_COUNT - CTL_RESTING - 1) * 4, s));
    DYN_CUDA(cudaMemsetAsync(dw.counters, 0, DYN_COUNTER_RESTING * 4, s));
    DYN_CUDA(cudaMemsetAsync(dw.counters + DYN_COUNTER_RESTING + 1, 0, (64 - DYN_COUNTER_RESTING - 1) * 4, s));
    // colliders may have moved between slots: no kept grid run survives a scene upload
    DYN_CUDA(cudaMemsetAsync(dw.c_held, 0, (size_t)d->k_cap * 4, s));
    DYN_CUDA(cudaMemsetAsync(dw.held, 0, HELD_COUNT * 4, s));
    DYN_CUDA(cudaStreamSynchronize(s));
    if ((st = upload_joints(w))) return st;
    w->scene_dirty = false;
    d->parity = 0;
    d->stepped = false;
    d->uploaded = true;
    d->scene_epoch += 1;
    release_graphs(d);
    return DYN_OK;
}

dyn_status download_states(dyn_world* w, std::vector<dyn_body_state_record>* out) {
    DeviceState* d = w->dev;
    uint32_t n = d->dw.n;
    out->resize(n);
    k_pack_states<<<blocks_for(d, std::max(n, 1u), 256), 256, 0, d->stream>>>(d->dw, d->staging, n);
    DYN_CUDA(cudaGetLastError());
    DYN_CUDA(cudaMemcpyAsync(out->data(), d->staging, (size_t)n * sizeof(dyn_body_state_record), cudaMemcpyDeviceToHost,
                             d->stream));
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    return DYN_OK;
}

// Stable LSD sort launches on `s` (see sort.cuh). Data ends in the primary buffers.
void record_sort(DeviceState* d, cudaStream_t s, uint32_t* major, uint32_t* minor, uint32_t* val, uint32_t* major_alt,
                 uint32_t* minor_alt, uint32_t* val_alt, const uint32_t* count_ptr, uint32_t n_fixed, uint32_t cap,
                 uint32_t major_digits, uint32_t minor_digits, uint32_t spin_limit = kLookbackSpinLimit,
                 uint32_t first_ticket = 0) {
    uint32_t passes = major_digits + minor_digits;
    if (passes == 0) return;
    uint32_t tiles = std::max(div_up(cap, kSortTile), 1u);
    cudaMemsetAsync(d->hist, 0, passes * 256 * 4, s);
    cudaMemsetAsync(d->tile_counters, 0, 16 * 4, s);
    if (first_ticket) {
        // test hook only: every pass's tickets start above tile 0, so the tiles after it wait on a
        // look-back word nothing writes until their bounded polls run out
        static uint32_t tickets[8];
        for (uint32_t& t : tickets) t = first_ticket;
        cudaMemcpyAsync(d->tile_counters, tickets, sizeof(tickets), cudaMemcpyHostToDevice, s);
    }
    cudaMemsetAsync(d->lookback, 0, (size_t)passes * tiles * 256 * 4, s);
    k_sort_histogram<<<std::min(div_up(cap, 256), d->sms * 4u), 256, 0, s>>>(major, minor, count_ptr, n_fixed, cap,
                                                                            (int)major_digits, (int)minor_digits, d->hist);
    k_sort_offsets<<<1, 256, 0, s>>>(d->hist, (int)passes);
    uint32_t* src_major = major;
    uint32_t* src_minor = minor;
    uint32_t* src_val = val;
    uint32_t* dst_major = major_alt;
    uint32_t* dst_minor = minor_alt;
    uint32_t* dst_val = val_alt;
    bool two = minor != nullptr;
    for (uint32_t p = 0; p < passes; ++p) {
        bool on_minor = p < minor_digits;
        int shift = 8 * (int)(on_minor ? p : p - minor_digits);
        uint32_t* key_in = on_minor ? src_minor : src_major;
        uint32_t* key_out = on_minor ? dst_minor : dst_major;
        uint32_t* oth_in = on_minor ? src_major : src_minor;
        uint32_t* oth_out = on_minor ? dst_major : dst_minor;
        uint32_t* lb = d->lookback + (size_t)p * tiles * 256;
        uint32_t* status = d->dw.ctl + CTL_STATUS;
        if (two && val) {
            k_onesweep<true, true><<<tiles, kSortThreads, 0, s>>>(key_in, oth_in, src_val, key_out, oth_out, dst_val, count_ptr,
                                                                   n_fixed, cap, shift, d->hist + p * 256, lb,
                                                                   d->tile_counters + p, status, spin_limit);
        } else if (two) {
            k_onesweep<true, false><<<tiles, kSortThreads, 0, s>>>(key_in, oth_in, nullptr, key_out, oth_out, nullptr, count_ptr,
                                                                    n_fixed, cap, shift, d->hist + p * 256, lb,
                                                                    d->tile_counters + p, status, spin_limit);
        } else if (val) {
            k_onesweep<false, true><<<tiles, kSortThreads, 0, s>>>(key_in, nullptr, src_val, key_out, nullptr, dst_val, count_ptr,
                                                                    n_fixed, cap, shift, d->hist + p * 256, lb,
                                                                    d->tile_counters + p, status, spin_limit);
        } else {
            k_onesweep<false, false><<<tiles, kSortThreads, 0, s>>>(key_in, nullptr, nullptr, key_out, nullptr, nullptr,
                                                                     count_ptr, n_fixed, cap, shift, d->hist + p * 256, lb,
                                                                     d->tile_counters + p, status, spin_limit);
        }
        std::swap(src_major, dst_major);
        std::swap(src_minor, dst_minor);
        std::swap(src_val, dst_val);
    }
    if (passes % 2 == 1) {
        // odd pass count: results sit in the alternate buffers
        size_t bytes = (size_t)cap * 4;
        cudaMemcpyAsync(major, src_major, bytes, cudaMemcpyDeviceToDevice, s);
        if (two) cudaMemcpyAsync(minor, src_minor, bytes, cudaMemcpyDeviceToDevice, s);
        if (val) cudaMemcpyAsync(val, src_val, bytes, cudaMemcpyDeviceToDevice, s);
    }
}

void record_scan(DeviceState* d, cudaStream_t s, const uint32_t* in, uint32_t* out, const uint32_t* count_ptr,
                 uint32_t n_fixed, uint32_t cap, uint32_t* total) {
    uint32_t tiles = std::max(div_up(cap, kSortTile), 1u);
    cudaMemsetAsync(d->tile_counters + 15, 0, 4, s);
    cudaMemsetAsync(d->lookback, 0, (size_t)tiles * 4, s);
    k_scan_exclusive<<<tiles, kSortThreads, 0, s>>>(in, out, count_ptr, n_fixed, cap, total, d->lookback, d->tile_counters + 15,
                                                    d->dw.ctl + CTL_STATUS, kLookbackSpinLimit);
}

struct Marker {
    DeviceState* d;
    cudaStream_t s;
    bool timed;
    void operator()(uint32_t stage) {
        if (!timed) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, s);
        d->events.push_back(e);
        d->event_stage.push_back(stage);
    }
};

// Does any body of the world declare continuous collision (the reference's CCD gate,
// crates/dynamis-rigid/src/domain.rs:85-96 from World::ccd_active, crates/dynamis-world/src/body.rs:503-514)?
bool world_has_ccd(const dyn_world* w) {
    for (const dyn_body_descriptor_record& desc : w->descs) {
        if (desc.flags & DYN_BODY_CCD) return true;
    }
    return false;
}

// Issues one step's kernels on `s`. parity selects which contact set is current. With a tape the
// step also snapshots what its adjoint needs into the tape's current slot (adjoint.cuh): the relay,
// k_solve and the fused position kernels write theirs as they run; the contact set and the body
// rows are copied by kernels of their own.
void record_step(dyn_world* w, cudaStream_t s, uint32_t parity, bool timed, const TapeView* tape = nullptr) {
    DeviceState* d = w->dev;
    DeviceWorld dw = d->dw;
    if (parity) std::swap(dw.cur, dw.arc);
    dw.solver_guard = w->solver_guard;
    if (tape) {
        dw.tape = TapeWrites{tape->slot, tape->relay, tape->vel, tape->acc, tape->res, tape->cnt,
                             tape->substeps, tape->iterations, tape->piterations, tape->n, tape->c};
    }
    const dyn_step_params p = d->params;
    Marker mark{d, s, timed};
    const uint32_t N = std::max(dw.n, 1u), K = std::max(dw.k, 1u), ND = std::max(dw.nd, 1u);
    const uint32_t E = dw.e_cap, P = dw.p_cap, C = dw.c_cap;
    const uint32_t joint_blocks = dw.jgroup_count;  // one warp group per 32-thread block
    // the frozen-contact store this step reads is the one the previous step's commit wrote
    dw.rest_cap = d->rest_cap;
    dw.rest_in = d->rest_ids[parity];
    dw.rest_in_slots = d->rest_slots[parity];
    dw.rest_out = d->rest_ids[1u - parity];
    dw.rest_out_slots = d->rest_slots[1u - parity];
    mark(ST_BEGIN);
    k_reset<<<1, 64, 0, s>>>(dw);
    if (dw.jcount) k_joint_count<<<blocks_for(d, std::max(dw.jfilter_count, 1u), 256), 256, 0, s>>>(dw);
    if (d->edit_graphs) {
        k_clear_inputs<<<blocks_for(d, N, 256), 256, 0, s>>>(dw);
        k_body_edits<<<blocks_for(d, std::max(d->edit_capacity, 1u), 128), 128, 0, s>>>(dw);
        k_begin<false><<<blocks_for(d, N, 256), 256, 0, s>>>(dw, p);
    } else {
        k_begin<true><<<blocks_for(d, N, 256), 256, 0, s>>>(dw, p);
    }
    mark(ST_AABB);
    k_aabb<<<blocks_for(d, K, 128), 128, 0, s>>>(dw, p);
    mark(ST_ENTRIES);
    // the awake run every step; the kept runs (immovable, resting) only when the gate finds them
    // stale, their scans and sorts otherwise covering nothing
    k_entry_count<true><<<blocks_for(d, K, 256), 256, 0, s>>>(dw);
    // one scan over the three runs' counts back to back; each run's key positions are its offsets
    // less the offset at the start of its third
    record_scan(d, s, dw.run_count, dw.run_offset, nullptr, 3 * dw.k, 3 * K, dw.held + HELD_SCRATCH);
    k_grid_gate<<<1, 32, 0, s>>>(dw);
    k_entry_emit<true><<<blocks_for(d, K, 256), 256, 0, s>>>(dw);
    mark(ST_ENTRY_SORT);
    for (uint32_t run = 0; run < 3; ++run) {
        const uint32_t* count = dw.held + (run == RUN_AWAKE ? HELD_AWAKE
                                           : run == RUN_IMMOVABLE ? HELD_SORT_IMMOVABLE : HELD_SORT_RESTING);
        record_sort(d, s, dw.run_key + (size_t)run * E, nullptr, dw.run_val + (size_t)run * E, dw.ekey_alt, nullptr,
                    dw.eval_alt, count, 0, E, 4, 0);
    }
    k_entry_merge<<<blocks_for(d, E, 256), 256, 0, s>>>(dw);
    mark(ST_PAIRS);
    k_cell_clear<<<blocks_for(d, 1u << dw.cell_bits, 256), 256, 0, s>>>(dw);
    k_cell_insert<<<blocks_for(d, E, 256), 256, 0, s>>>(dw);
    // Independent kernels run as parallel branches of the captured graph (a fork onto the side
    // stream and a join back): the coarse links beside the same-cell scan, the analytic classes
    // beside the convex chain. They only share append counters, and every product they feed is
    // sorted or order-independent. The eager timed path keeps one stream, so stage times stay apart.
    const bool branches = !timed;
    cudaStream_t side = branches ? d->side_stream : s;
    cudaStream_t side2 = branches ? d->side_stream2 : s;
    auto fork = [&](uint32_t k, cudaStream_t to) {
        if (!branches) return;
        cudaEventRecord(d->fork_events[k], s);
        cudaStreamWaitEvent(to, d->fork_events[k], 0);
    };
    auto join = [&](uint32_t k, cudaStream_t from) {
        if (!branches) return;
        cudaEventRecord(d->join_events[k], from);
        cudaStreamWaitEvent(s, d->join_events[k], 0);
    };
    fork(0, side);
    k_pairs_coarse<<<dim3(blocks_for(d, K, 128), kCoarseLevelSlices), 128, 0, s>>>(dw);
    k_pairs_cell<<<blocks_for(d, E, 256), 256, 0, side>>>(dw);
    join(0, side);
    // the candidate pairs stay in emission order; the contacts are sorted into pair order below
    mark(ST_NARROWPHASE);
    k_pair_class<<<blocks_for(d, P, 256), 256, 0, s>>>(dw);
    fork(1, side);
    k_narrow_class<PC_ANALYTIC><<<blocks_for(d, P, 128), 128, 0, side>>>(dw, p);
    k_narrow_class<PC_BOXES><<<blocks_for(d, P, 128), 128, 0, side>>>(dw, p);
    k_convex_reject<<<blocks_for(d, P, 128), 128, 0, s>>>(dw, p);
    // persistent: lanes draw pairs from a ticket; six blocks per SM is the occupancy its registers allow
    k_convex_gjk<<<d->sms * d->launch.gjk_blocks_per_sm, 128, 0, s>>>(dw, p);
    // separated pairs (probe) and penetrating ones (EPA) are disjoint queues
    fork(3, side2);
    k_convex_probe<<<blocks_for(d, P, 128), 128, 0, side2>>>(dw, p);
    k_convex_epa<<<d->sms * d->launch.epa_blocks_per_sm, 32 * kEpaWarpsPerBlock, 0, s>>>(dw, p);
    join(3, side2);
    k_convex_manifold<<<blocks_for(d, P, 128), 128, 0, s>>>(dw, p);
    join(1, side);
    mark(ST_COMPACT);
    k_contact_keys<<<blocks_for(d, C, 256), 256, 0, s>>>(dw);
    const uint32_t words = key_words(std::max(dw.k, 1u));
    record_sort(d, s, dw.cmaj, dw.cmin, dw.cval, dw.cmaj_alt, dw.cmin_alt, dw.cval_alt, dw.ctl + CTL_STAGED, 0, dw.s_cap, words,
                words);
    k_contact_gather<<<blocks_for(d, C, 128), 128, 0, s>>>(dw);
    // the solver blocks (target speeds, row claims) beside the identity, islands and wake passes:
    // neither reads what the other writes (the relay rewrites only the w word of a contact's rows
    // and the carried impulses; waking clears sleep flags the row claims do not look at)
    mark(ST_SOLVER_PREPARE);
    fork(2, side);
    k_solver_blocks<<<blocks_for(d, C, 256), 256, 0, side>>>(dw, p);
    record_scan(d, side, dw.row_flag, dw.row_offset, nullptr, std::max(dw.n, 1u), N, dw.ctl + CTL_SOLVER_ROWS);
    k_solver_row_list<<<blocks_for(d, N, 256), 256, 0, side>>>(dw);
    mark(ST_IDENTITY);
    if (tape) k_tape_clear_relay<<<blocks_for(d, 4 * C, 256), 256, 0, s>>>(*tape);
    k_relay<<<blocks_for(d, C, 128), 128, 0, s>>>(dw);
    k_contact_begin<<<blocks_for(d, C, 256), 256, 0, s>>>(dw, p);
    mark(ST_ISLANDS);
    k_island_link<true><<<blocks_for(d, C, 256), 256, 0, s>>>(dw, p);
    k_island_flatten<false><<<blocks_for(d, ND, 256), 256, 0, s>>>(dw);
    k_island_link<false><<<blocks_for(d, C, 256), 256, 0, s>>>(dw, p);
    if (dw.jcount) k_island_link_joints<<<blocks_for(d, dw.jcount, 256), 256, 0, s>>>(dw);
    k_island_flatten<true><<<blocks_for(d, ND, 256), 256, 0, s>>>(dw);
    mark(ST_WAKE_LIVE);
    k_wake_live<<<blocks_for(d, ND, 256), 256, 0, s>>>(dw);
    join(2, side);
    if (tape) k_tape_contacts<<<blocks_for(d, C, 256), 256, 0, s>>>(dw, *tape);
    for (uint32_t sub = 0; sub < p.substeps; ++sub) {
        mark(ST_INTEGRATE);
        if (tape) k_tape_hot<<<blocks_for(d, N, 256), 256, 0, s>>>(dw, *tape, sub);
        k_integrate<<<blocks_for(d, N, 256), 256, 0, s>>>(dw, p);
        const uint32_t st = d->launch.solve_threads;
        k_solve_prepare<<<blocks_for(d, C, st), st, 0, s>>>(dw);
        if (sub == 0) {
            mark(ST_WARM);
            if (joint_blocks) k_joints<JP_WARM><<<joint_blocks, 32, 0, s>>>(dw, p);
            k_warm<<<blocks_for(d, C, st), st, 0, s>>>(dw);
            k_vapply<<<blocks_for(d, N, 256), 256, 0, s>>>(dw);
        }
        mark(ST_VELOCITY);
        for (uint32_t it = 0; it < p.solve_iterations; ++it) {
            if (joint_blocks) k_joints<JP_SOLVE><<<joint_blocks, 32, 0, s>>>(dw, p);
            k_solve<<<blocks_for(d, C, st), st, 0, s>>>(dw, p, sub * p.solve_iterations + it);
            k_vapply<<<blocks_for(d, N, 256), 256, 0, s>>>(dw);
        }
        mark(ST_ADVANCE);
        k_advance<<<blocks_for(d, N, 256), 256, 0, s>>>(dw, p);
        mark(ST_POSITION);
        if (joint_blocks == 0u) {
            // each iteration applies the one before it; one apply after the last
            for (uint32_t it = 0; it < p.position_iterations; ++it) {
                if (it == 0u) {
                    k_position_fused<true><<<blocks_for(d, C, st), st, 0, s>>>(dw, p, it, sub);
                } else {
                    k_position_fused<false><<<blocks_for(d, C, st), st, 0, s>>>(dw, p, it, sub);
                }
            }
            if (p.position_iterations > 0u) {
                k_papply_last<<<blocks_for(d, N, 256), 256, 0, s>>>(dw, p.position_iterations, sub);
            }
        } else {
            for (uint32_t it = 0; it < p.position_iterations; ++it) {
                k_joints<JP_POSITION><<<joint_blocks, 32, 0, s>>>(dw, p);
                k_position<<<blocks_for(d, C, 256), 256, 0, s>>>(dw, p);
                k_papply<<<blocks_for(d, N, 256), 256, 0, s>>>(dw);
            }
        }
    }
    if (world_has_ccd(w)) {
        // continuous collision of the bodies that declare it (ccd.cuh): sweep, pick, impact, retreat
        mark(ST_CCD);
        k_ccd_sweep<<<blocks_for(d, P, 128), 128, 0, s>>>(dw, p);
        k_ccd_pick<<<blocks_for(d, 2 * P, 256), 256, 0, s>>>(dw);
        k_ccd_impact<<<blocks_for(d, 2 * P, 256), 256, 0, s>>>(dw);
        k_ccd_apply<<<blocks_for(d, N, 256), 256, 0, s>>>(dw);
    }
    mark(ST_SLEEP);
    k_sleep<<<blocks_for(d, ND, 256), 256, 0, s>>>(dw, p);
    // commit (crates/dynamis-rigid/src/commit.rs:187-208): thaw with the static wake flags, freeze
    k_rest_thaw<<<blocks_for(d, std::max(dw.rest_cap, N), 256), 256, 0, s>>>(dw);
    k_rest_freeze<<<blocks_for(d, C, 256), 256, 0, s>>>(dw);
    k_rest_commit<<<1, 32, 0, s>>>(dw);
    if (tape) {
        k_tape_hot<<<blocks_for(d, N, 256), 256, 0, s>>>(dw, *tape, p.substeps);
        k_tape_advance<<<1, 32, 0, s>>>(*tape);
    }
    mark(ST_COUNT);
}

// The queued body edits as runs of one row each (command order within a row, rows in order of
// their first edit, as command.rs:157-176 compiles them), onto the device for the next step.
dyn_status upload_edits(dyn_world* w) {
    DeviceState* d = w->dev;
    DeviceWorld& dw = d->dw;
    const uint32_t n = (uint32_t)w->edits.size();
    if (n == 0) {
        if (d->edits_pending_on_device) {
            DYN_CUDA(cudaMemsetAsync(dw.edit_count, 0, 4, d->stream));
            d->edits_pending_on_device = false;
        }
        return DYN_OK;
    }
    std::vector<uint32_t> order;  // edit indices grouped by row
    std::vector<uint4> runs;
    {
        std::vector<uint32_t> rows(n);
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t id = w->edit_ids[i];
            rows[i] = id < w->row_of_id.size() ? w->row_of_id[id] : DYN_NO_BODY;
        }
        std::vector<uint32_t> run_of_row;  // row -> run index + 1
        std::vector<std::vector<uint32_t>> members;
        std::vector<uint32_t> run_rows;
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t row = rows[i];
            if (row == DYN_NO_BODY || row >= w->states.size()) continue;
            if (run_of_row.size() <= row) run_of_row.resize(row + 1, 0u);
            if (run_of_row[row] == 0u) {
                members.emplace_back();
                run_rows.push_back(row);
                run_of_row[row] = (uint32_t)members.size();
            }
            members[run_of_row[row] - 1].push_back(i);
        }
        for (size_t r = 0; r < members.size(); ++r) {
            runs.push_back(make_uint4(run_rows[r], (uint32_t)order.size(), (uint32_t)members[r].size(), 0u));
            order.insert(order.end(), members[r].begin(), members[r].end());
        }
    }
    std::vector<dyn_body_edit_record> grouped(order.size());
    for (size_t i = 0; i < order.size(); ++i) grouped[i] = w->edits[order[i]];
    w->edits.clear();
    w->edit_ids.clear();
    const uint32_t need = std::max((uint32_t)grouped.size(), (uint32_t)runs.size());
    if (need > d->edit_capacity || !d->edit_graphs) {
        uint32_t cap = std::max(need, std::max(2 * d->edit_capacity, 256u));
        DYN_CUDA(cudaStreamSynchronize(d->stream));
        if (d->edit_buffer) cudaFree(d->edit_buffer);
        if (d->edit_run_buffer) cudaFree(d->edit_run_buffer);
        d->edit_buffer = nullptr;
        d->edit_run_buffer = nullptr;
        DYN_CUDA(cudaMalloc(&d->edit_buffer, (size_t)cap * sizeof(dyn_body_edit_record)));
        DYN_CUDA(cudaMalloc(&d->edit_run_buffer, (size_t)cap * sizeof(uint4)));
        d->edit_capacity = cap;
        dw.edits = d->edit_buffer;
        dw.edit_runs = d->edit_run_buffer;
        d->edit_graphs = true;
        release_graphs(d);  // the step graph gains the edit kernels and the new buffers
    }
    uint32_t count = (uint32_t)runs.size();
    if (!grouped.empty()) {
        DYN_CUDA(cudaMemcpyAsync(d->edit_buffer, grouped.data(), grouped.size() * sizeof(dyn_body_edit_record),
                                 cudaMemcpyHostToDevice, d->stream));
    }
    if (count) {
        DYN_CUDA(cudaMemcpyAsync(d->edit_run_buffer, runs.data(), runs.size() * sizeof(uint4), cudaMemcpyHostToDevice,
                                 d->stream));
    }
    DYN_CUDA(cudaMemcpyAsync(dw.edit_count, &count, 4, cudaMemcpyHostToDevice, d->stream));
    DYN_CUDA(cudaStreamSynchronize(d->stream));  // the host vectors above go out of scope
    d->edits_pending_on_device = count != 0;
    return DYN_OK;
}

dyn_status prepare_step(dyn_world* w, float dt) {
    if (!(dt > 0.0f) || !std::isfinite(dt)) return fail(w, DYN_ERR_INVALID, "a step timestep must be positive");
    bool fresh = !w->dev || !w->dev->uploaded || (w->rows_dirty && !w->raw_rows) || w->scene_dirty;
    if (fresh || w->joints_dirty) {
        dyn_status st = save_joint_runtime(w);
        if (st) return st;
    }
    if (fresh) {
        // bodies spawned or removed after stepping: keep the simulated states of the others
        dyn_status st = sync_spawn_states(w);
        if (st) return st;
    }
    if (fresh) {
        dyn_status st = upload_scene(w);
        if (st) return st;
    } else if (w->joints_dirty) {
        dyn_status st = upload_joints(w);
        if (st) return st;
    }
    if (w->states.empty()) return fail(w, DYN_ERR_INVALID, "the world holds no bodies");
    DeviceState* d = w->dev;
    if (dyn_status st = upload_edits(w)) return st;
    dyn_step_params p;
    dyn_step_params_for(w, dt, &p);
    if (d->graph_dt != dt) {
        release_graphs(d);
        d->params = p;
        d->graph_dt = dt;
    }
    return DYN_OK;
}

}  // namespace

// ---- observation ring ----
void release_observer(dyn_world* w) {
    Observer& o = w->observer;
    for (ObservationSlot& s : o.slots) {
        if (s.done) cudaEventSynchronize(static_cast<cudaEvent_t>(s.done));
        if (s.states) cudaFreeHost(s.states);
        if (s.counters) cudaFreeHost(s.counters);
        if (s.done) cudaEventDestroy(static_cast<cudaEvent_t>(s.done));
        s = ObservationSlot();
    }
    if (o.ids_dev) cudaFree(o.ids_dev);
    o.ids_dev = nullptr;
    o.ids_dev_capacity = 0;
    o.ids_dirty = true;
    o.latest = -1;
}
// World::poll: every slot whose copies have completed becomes readable; the newest is the latest.
void observer_poll(dyn_world* w) {
    Observer& o = w->observer;
    for (uint32_t i = 0; i < kObservationSlots; ++i) {
        ObservationSlot& s = o.slots[i];
        if (!s.pending) continue;
        cudaError_t e = cudaEventQuery(static_cast<cudaEvent_t>(s.done));
        if (e == cudaErrorNotReady) continue;
        cudaGetLastError();
        s.pending = false;
        s.ready = e == cudaSuccess;
        if (s.ready && (o.latest < 0 || s.step > o.slots[o.latest].step)) o.latest = (int)i;
    }
}
// After a step: copy the observed records and the counters into a slot other than the latest
// (which a reader may be copying from): a completed one if there is one, else the oldest still in
// flight, whose copy this newer one supersedes (the copies are ordered on the stream, so the new one
// lands after it; the host never reads a slot in flight).
dyn_status observe_after_step(dyn_world* w) {
    Observer& o = w->observer;
    DeviceState* d = w->dev;
    observer_poll(w);
    int pick = -1;
    for (uint32_t k = 0; k < kObservationSlots; ++k) {
        if (!o.slots[k].pending && (int)k != o.latest) {
            pick = (int)k;
            break;
        }
    }
    if (pick < 0) {
        for (uint32_t k = 0; k < kObservationSlots; ++k) {
            if ((int)k == o.latest) continue;
            if (pick < 0 || o.slots[k].step < o.slots[pick].step) pick = (int)k;
        }
        o.superseded += 1;
    }
    ObservationSlot& s = o.slots[pick];
    s.index_of_id.clear();
    const uint32_t m = o.all ? (uint32_t)w->states.size() : (uint32_t)o.ids.size();
    if (!o.all && o.ids_dirty) {
        // the observed set changed (dyn_observe_bodies): one synchronous upload, then none per step
        if (m > o.ids_dev_capacity) {
            if (o.ids_dev) cudaFree(o.ids_dev);
            o.ids_dev = nullptr;
            o.ids_dev_capacity = 0;
            DYN_CUDA(cudaMalloc(&o.ids_dev, (size_t)std::max(m, 1u) * 4));
            o.ids_dev_capacity = std::max(m, 1u);
        }
        if (m > 0) DYN_CUDA(cudaMemcpy(o.ids_dev, o.ids.data(), (size_t)m * 4, cudaMemcpyHostToDevice));
        o.ids_dirty = false;
    }
    if (m > s.capacity) {
        if (s.states) cudaFreeHost(s.states);
        s.states = nullptr;
        s.capacity = 0;
        DYN_CUDA(cudaHostAlloc(&s.states, (size_t)std::max(m, 1u) * sizeof(dyn_body_state_record), cudaHostAllocDefault));
        s.capacity = std::max(m, 1u);
    }
    if (!s.counters) DYN_CUDA(cudaHostAlloc(&s.counters, 64 * sizeof(uint32_t), cudaHostAllocDefault));
    if (!s.done) {
        cudaEvent_t e;
        DYN_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        s.done = e;
    }
    if (m > 0) {
        if (o.all) {
            k_pack_states<<<blocks_for(d, m, 256), 256, 0, d->stream>>>(d->dw, d->staging, m);
        } else {
            k_pack_ids<<<blocks_for(d, m, 256), 256, 0, d->stream>>>(d->dw, static_cast<const uint32_t*>(o.ids_dev),
                                                                 d->staging, m);
        }
        DYN_CUDA(cudaGetLastError());
        DYN_CUDA(cudaMemcpyAsync(s.states, d->staging, (size_t)m * sizeof(dyn_body_state_record), cudaMemcpyDeviceToHost,
                                 d->stream));
    }
    DYN_CUDA(cudaMemcpyAsync(s.counters, d->dw.counters, 64 * sizeof(uint32_t), cudaMemcpyDeviceToHost, d->stream));
    DYN_CUDA(cudaEventRecord(static_cast<cudaEvent_t>(s.done), d->stream));
    s.count = m;
    s.step = w->steps_taken;
    s.pending = true;
    s.ready = false;
    return DYN_OK;
}

dyn_status sync_spawn_states(dyn_world* w) {
    if (!w->dev || !w->dev->stepped || w->raw_rows) return DYN_OK;
    std::vector<dyn_body_state_record> now;
    dyn_status st = download_states(w, &now);
    if (st) return st;
    for (const dyn_body_state_record& s : now) {
        if (s.body_id < w->spawn_states.size()) w->spawn_states[s.body_id] = s;
    }
    return DYN_OK;
}

void destroy_device(dyn_world* w) {
    DeviceState* d = w->dev;
    if (!d) return;
    cudaSetDevice(w->device);
    // the caller's stream may already be gone: wait for the whole device instead
    cudaDeviceSynchronize();
    release_graphs(d);
    free_tape_memory(d);
    for (cudaEvent_t e : d->events) cudaEventDestroy(e);
    for (void* p : d->allocs) cudaFree(p);
    if (d->spill_host) cudaFreeHost(d->spill_host);
    for (void* p : d->joint_allocs) cudaFree(p);
    if (d->edit_buffer) cudaFree(d->edit_buffer);
    if (d->edit_run_buffer) cudaFree(d->edit_run_buffer);
    if (d->query_buf) cudaFree(d->query_buf);
    if (d->hit_buf) cudaFree(d->hit_buf);
    if (d->query_entries) cudaFree(d->query_entries);
    if (d->query_words) cudaFree(d->query_words);
    for (uint32_t* p : {d->sort_alt0, d->sort_alt1, d->sort_alt2}) {
        if (p) cudaFree(p);
    }
    for (uint32_t i = 0; i < 4; ++i) {
        if (d->fork_events[i]) cudaEventDestroy(d->fork_events[i]);
        if (d->join_events[i]) cudaEventDestroy(d->join_events[i]);
        if (d->inflight[i]) cudaEventDestroy(d->inflight[i]);
    }
    if (d->side_stream) cudaStreamDestroy(d->side_stream);
    if (d->side_stream2) cudaStreamDestroy(d->side_stream2);
    if (d->own_stream) cudaStreamDestroy(d->own_stream);
    delete d;
    w->dev = nullptr;
    cudaGetLastError();  // nothing from tear-down may surface in a later, unrelated call
}

}  // namespace dyn

using namespace dyn;

extern "C" {

DYN_API dyn_status dyn_world_create(const dyn_config* config, const dyn_capacity* capacity, int32_t device, dyn_world** out) {
    if (!out) return DYN_ERR_INVALID;
    *out = nullptr;
    dyn_world* w = new dyn_world();
    if (config) {
        w->config = *config;
    } else {
        dyn_config_default(&w->config);
    }
    if (capacity) w->capacity = *capacity;
    w->device = device;
    const dyn_config& c = w->config;
    if (c.substeps == 0 || c.solve_iterations == 0 || !(c.slop >= 0.0f) || !(c.contact_margin >= 0.0f)
        || !(c.sleep_time > 0.0f) || c.friction_combine > 3 || c.restitution_combine > 3) {
        delete w;
        return DYN_ERR_INVALID;
    }
    *out = w;
    return DYN_OK;
}

DYN_API dyn_status dyn_world_destroy(dyn_world* w) {
    if (!w) return DYN_ERR_INVALID;
    if (w->dev) cudaSetDevice(w->device);
    release_observer(w);
    destroy_device(w);
    delete w;
    return DYN_OK;
}

DYN_API dyn_status dyn_world_set_stream(dyn_world* w, void* stream) {
    if (!w) return DYN_ERR_INVALID;
    if (!w->dev) {
        dyn_status st = ensure_device(w);
        if (st) return st;
    }
    w->user_stream = stream;
    w->dev->stream = stream ? static_cast<cudaStream_t>(stream) : w->dev->own_stream;
    return DYN_OK;
}

DYN_API dyn_status dyn_upload_bodies(dyn_world* w, const dyn_body_state_record* states, const dyn_body_descriptor_record* descs,
                                     uint32_t n, const dyn_collider_record* colliders, const uint32_t* owners, uint32_t k) {
    if (!w || (n && (!states || !descs)) || (k && (!colliders || !owners)))
        return fail(w, DYN_ERR_INVALID, "dyn_upload_bodies: null argument");
    uint32_t dynamic = 0;
    bool prefix = true;
    for (uint32_t i = 0; i < n; ++i) {
        bool dyn_row = (descs[i].flags & DYN_BODY_KINEMATIC) == 0u && descs[i].inverse_mass > 0.0f;
        if (dyn_row) {
            if (!prefix) return fail(w, DYN_ERR_INVALID, "dyn_upload_bodies: dynamic rows must come first");
            ++dynamic;
        } else {
            prefix = false;
        }
    }
    for (uint32_t i = 0; i < k; ++i) {
        if (owners[i] != DYN_NO_BODY && owners[i] >= n) return fail(w, DYN_ERR_INVALID, "dyn_upload_bodies: owner out of range");
        if (colliders[i].kind == DYN_SHAPE_HULL && colliders[i].source >= w->hulls.size())
            return fail(w, DYN_ERR_INVALID, "dyn_upload_bodies: unknown hull source");
    }
    w->raw_rows = true;
    w->rows_dirty = false;
    w->states.assign(states, states + n);
    w->descs.assign(descs, descs + n);
    w->colliders.assign(colliders, colliders + k);
    w->owners.assign(owners, owners + k);
    w->dynamic_count = dynamic;
    uint32_t max_id = 0;
    for (uint32_t i = 0; i < n; ++i) max_id = std::max(max_id, states[i].body_id + 1);
    w->row_of_id.assign(std::max(max_id, n), DYN_NO_BODY);
    for (uint32_t i = 0; i < n; ++i) w->row_of_id[states[i].body_id] = i;
    w->body_world.assign(n, 0u);
    for (uint32_t i = 0; i < n; ++i) {
        if (states[i].body_id < w->world_of_id.size()) w->body_world[i] = w->world_of_id[states[i].body_id];
    }
    return upload_scene(w);
}

DYN_API dyn_status dyn_upload_states(dyn_world* w, const dyn_body_state_record* states, uint32_t n) {
    if (!w || !states) return fail(w, DYN_ERR_INVALID, "dyn_upload_states: null argument");
    rebuild_rows(w);
    if (n != w->states.size()) return fail(w, DYN_ERR_INVALID, "dyn_upload_states: row count differs from the scene");
    if (!w->dev || !w->dev->uploaded || (w->rows_dirty && !w->raw_rows) || w->scene_dirty) {
        dyn_status st = upload_scene(w);
        if (st) return st;
    }
    DeviceState* d = w->dev;
    // one contiguous copy of the ABI records, then a kernel scatters them into the device layout
    DYN_CUDA(cudaMemcpyAsync(d->staging, states, (size_t)n * sizeof(dyn_body_state_record), cudaMemcpyHostToDevice,
                             d->stream));
    k_unpack_states<<<blocks_for(d, std::max(n, 1u), 256), 256, 0, d->stream>>>(d->dw, d->staging, n);
    DYN_CUDA(cudaGetLastError());
    return DYN_OK;
}

// The pair stream widens after a step that refused pairs, as the reference widens its streams
// after a spill (crates/dynamis-broadphase/src/capacity.rs:27-80 plans the pair stream from the
// measured pair count; crates/dynamis-world/tests/suite/capacity.rs:142-187: within a few steps
// the step stops refusing). Every step's last kernel leaves the pair demand and any refusal in
// host-mapped memory, and each dyn_step reads them without waiting. Up to kStepsInFlight steps
// are queued ahead of the device, so a refusal is seen up to that many steps after it happened;
// the stream therefore also widens as soon as the demand passes half of it, which keeps a growing
// pile from reaching the limit before the host sees it. The new size is grown() of
// crates/dynamis-domain/src/capacity.rs:15-23 applied to twice the demand: at least twice the
// stream. The pair buffers are per-step scratch: nothing in them outlives a step, so they are
// replaced, not copied. If the wider buffers cannot be had, the stream keeps its size and the
// refusals stay counted.
constexpr uint64_t kMaxPairCapacity = 1ull << 27;
constexpr uint32_t kStepsInFlight = 4u;
dyn_status widen_pair_stream(dyn_world* w) {
    DeviceState* d = w->dev;
    volatile uint32_t* mail = d->spill_host;
    if (!mail || d->p_cap >= kMaxPairCapacity) return DYN_OK;
    if (mail[2] == 0u && mail[1] <= d->p_cap / 2) return DYN_OK;
    DYN_CUDA(cudaStreamSynchronize(d->stream));  // no step in flight writes the mailbox or the buffers
    const uint64_t demand = mail[1];
    mail[1] = 0u;
    mail[2] = 0u;
    uint64_t want = std::max<uint64_t>(2ull * demand, 2ull * d->p_cap);
    want = std::min<uint64_t>((want + 1023u) & ~1023ull, kMaxPairCapacity);
    if (want <= d->p_cap) return DYN_OK;
    const size_t P = (size_t)want;
    DeviceWorld& dw = d->dw;
    struct Buffer {
        void** slot;
        size_t bytes;
        void* fresh;
    };
    Buffer list[] = {{reinterpret_cast<void**>(&dw.pmaj), P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&dw.pmin), P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&dw.np_list), (PC_COUNT + 1) * P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&dw.epa_list), P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&dw.epa_simplex), 4 * P * sizeof(float4), nullptr},
                     {reinterpret_cast<void**>(&dw.probe_list), P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&dw.probe_data), 6 * P * sizeof(float4), nullptr},
                     {reinterpret_cast<void**>(&dw.hit_list), P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&dw.hit_data), 2 * P * sizeof(float4), nullptr},
                     // the staging set of the narrowphase's contacts (one per pair at most) and its sort
                     {reinterpret_cast<void**>(&dw.tmp.normal), P * sizeof(float4), nullptr},
                     {reinterpret_cast<void**>(&dw.tmp.rows), P * sizeof(uint4), nullptr},
                     {reinterpret_cast<void**>(&dw.tmp.mat), P * sizeof(float4), nullptr},
                     {reinterpret_cast<void**>(&dw.tmp.ids), P * sizeof(uint4), nullptr},
                     {reinterpret_cast<void**>(&dw.tmp.ids2), P * sizeof(uint4), nullptr},
                     {reinterpret_cast<void**>(&dw.tmp.extra), P * sizeof(float4), nullptr},
                     {reinterpret_cast<void**>(&dw.tmp.la), 4 * P * sizeof(float4), nullptr},
                     {reinterpret_cast<void**>(&dw.tmp.lb), 4 * P * sizeof(float4), nullptr},
                     {reinterpret_cast<void**>(&dw.tmp.acc), 4 * P * sizeof(float4), nullptr},
                     {reinterpret_cast<void**>(&dw.tmp.pos), 4 * P * sizeof(float4), nullptr},
                     {reinterpret_cast<void**>(&dw.cmaj), P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&dw.cmin), P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&dw.cval), P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&dw.cmaj_alt), P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&dw.cmin_alt), P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&dw.cval_alt), P * sizeof(uint32_t), nullptr},
                     {reinterpret_cast<void**>(&d->lookback),
                      (size_t)8 * std::max(div_up(std::max<size_t>(d->e_cap, P), kSortTile), 1u) * 256 * sizeof(uint32_t), nullptr}};
    for (Buffer& b : list) {
        if (cudaMalloc(&b.fresh, b.bytes) != cudaSuccess) {
            for (Buffer& f : list) if (f.fresh) cudaFree(f.fresh);
            (void)cudaGetLastError();  // out of memory: keep the stream, keep counting refusals
            return DYN_OK;
        }
    }
    for (Buffer& b : list) {
        auto it = std::find(d->allocs.begin(), d->allocs.end(), *b.slot);
        if (it != d->allocs.end()) d->allocs.erase(it);
        DYN_CUDA(cudaFree(*b.slot));
        DYN_CUDA(cudaMemsetAsync(b.fresh, 0, b.bytes, d->stream));
        d->allocs.push_back(b.fresh);
        *b.slot = b.fresh;
    }
    d->p_cap = dw.p_cap = dw.s_cap = (uint32_t)P;
    d->lookback_words = (size_t)8 * std::max(div_up(std::max<size_t>(d->e_cap, P), kSortTile), 1u) * 256;
    release_graphs(d);  // the graphs hold the old buffers and capacity
    return DYN_OK;
}

// The contact stream widens like the pair stream (crates/dynamis-broadphase/src/capacity.rs:27-90
// grows every stream from its demand): once a step staged more contacts than the stream holds, or
// more than three quarters of it, the next dyn_step waits for the queued steps and replaces the contact sets
// and the solver's per-contact buffers with ones for twice the demand (at least twice the stream).
// The archived set, which the next step's relay reads, is copied over with the new point stride.
// Not while a tape is recording: its slots and checkpoints keep the stream's layout.
constexpr uint64_t kMaxContactCapacity = 1ull << 26;
dyn_status widen_contact_stream(dyn_world* w) {
    DeviceState* d = w->dev;
    volatile uint32_t* mail = d->spill_host;
    if (!mail || d->c_cap >= kMaxContactCapacity || d->tape.active || d->tuning) return DYN_OK;
    if (mail[3] <= d->c_cap - d->c_cap / 4) return DYN_OK;
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    const uint64_t demand = mail[3];
    mail[3] = 0u;
    uint64_t want = std::max<uint64_t>(2ull * demand, 2ull * d->c_cap);
    want = std::min<uint64_t>((want + 1023u) & ~1023ull, kMaxContactCapacity);
    if (want <= d->c_cap) return DYN_OK;
    const size_t C = (size_t)want, old = d->c_cap;
    DeviceWorld& dw = d->dw;
    ContactSet fresh_cur{}, fresh_arc{};
    SolverRows fresh_rows{};
    uint32_t *matched = nullptr, *cowner = nullptr;
    std::vector<void*> made;
    auto grab = [&](auto** ptr, size_t bytes) -> bool {
        void* q = nullptr;
        if (cudaMalloc(&q, bytes) != cudaSuccess) return false;
        made.push_back(q);
        *ptr = static_cast<std::remove_reference_t<decltype(**ptr)>*>(q);
        return true;
    };
    bool ok = true;
    for (ContactSet* set : {&fresh_cur, &fresh_arc}) {
        ok = ok && grab(&set->normal, C * sizeof(float4)) && grab(&set->rows, C * sizeof(uint4)) &&
             grab(&set->mat, C * sizeof(float4)) && grab(&set->ids, C * sizeof(uint4)) && grab(&set->ids2, C * sizeof(uint4)) &&
             grab(&set->extra, C * sizeof(float4)) && grab(&set->la, 4 * C * sizeof(float4)) &&
             grab(&set->lb, 4 * C * sizeof(float4)) && grab(&set->acc, 4 * C * sizeof(float4)) &&
             grab(&set->pos, 4 * C * sizeof(float4));
    }
    ok = ok && grab(&fresh_rows.arm_a, 4 * C * sizeof(float4)) && grab(&fresh_rows.arm_b, 4 * C * sizeof(float4)) &&
         grab(&fresh_rows.masses, 4 * C * sizeof(float4)) && grab(&fresh_rows.tangent1, C * sizeof(float4)) &&
         grab(&fresh_rows.tangent2, C * sizeof(float4)) && grab(&matched, C * sizeof(uint32_t)) &&
         grab(&cowner, C * sizeof(uint32_t));
    if (!ok) {
        for (void* q : made) cudaFree(q);
        (void)cudaGetLastError();  // out of memory: keep the stream, keep counting refusals
        return DYN_OK;
    }
    for (void* q : made) DYN_CUDA(cudaMemsetAsync(q, 0, 1, d->stream));  // (contents are written before read)
    // the set the next step archives from: dw.arc at parity 0, dw.cur at parity 1 (record_step swaps)
    const ContactSet& archived = d->parity == 0u ? dw.arc : dw.cur;
    ContactSet& target = d->parity == 0u ? fresh_arc : fresh_cur;
    const uint32_t count = std::min<uint32_t>((uint32_t)old, 0xFFFFFFFFu);
    auto copy = [&](void* to, const void* from, size_t bytes) -> cudaError_t {
        return cudaMemcpyAsync(to, from, bytes, cudaMemcpyDeviceToDevice, d->stream);
    };
    DYN_CUDA(copy(target.normal, archived.normal, count * sizeof(float4)));
    DYN_CUDA(copy(target.rows, archived.rows, count * sizeof(uint4)));
    DYN_CUDA(copy(target.mat, archived.mat, count * sizeof(float4)));
    DYN_CUDA(copy(target.ids, archived.ids, count * sizeof(uint4)));
    DYN_CUDA(copy(target.ids2, archived.ids2, count * sizeof(uint4)));
    DYN_CUDA(copy(target.extra, archived.extra, count * sizeof(float4)));
    for (size_t pt = 0; pt < 4; ++pt) {  // point slot pt of contact i sits at pt * capacity + i
        DYN_CUDA(copy(target.la + pt * C, archived.la + pt * old, count * sizeof(float4)));
        DYN_CUDA(copy(target.lb + pt * C, archived.lb + pt * old, count * sizeof(float4)));
        DYN_CUDA(copy(target.acc + pt * C, archived.acc + pt * old, count * sizeof(float4)));
        DYN_CUDA(copy(target.pos + pt * C, archived.pos + pt * old, count * sizeof(float4)));
    }
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    std::vector<void*> stale = {dw.cur.normal, dw.cur.rows, dw.cur.mat, dw.cur.ids, dw.cur.ids2, dw.cur.extra, dw.cur.la,
                                dw.cur.lb, dw.cur.acc, dw.cur.pos, dw.arc.normal, dw.arc.rows, dw.arc.mat, dw.arc.ids,
                                dw.arc.ids2, dw.arc.extra, dw.arc.la, dw.arc.lb, dw.arc.acc, dw.arc.pos, dw.srows.arm_a,
                                dw.srows.arm_b, dw.srows.masses, dw.srows.tangent1, dw.srows.tangent2, dw.matched, dw.cowner};
    for (void* q : stale) {
        auto it = std::find(d->allocs.begin(), d->allocs.end(), q);
        if (it != d->allocs.end()) d->allocs.erase(it);
        DYN_CUDA(cudaFree(q));
    }
    for (void* q : made) d->allocs.push_back(q);
    dw.cur = fresh_cur;
    dw.arc = fresh_arc;
    dw.srows = fresh_rows;
    dw.matched = matched;
    dw.cowner = cowner;
    d->c_cap = dw.c_cap = (uint32_t)C;
    release_graphs(d);
    return DYN_OK;
}

DYN_API dyn_status dyn_stream_capacity(const dyn_world* w, uint32_t* pairs, uint32_t* contacts) {
    if (!w || !pairs || !contacts) return DYN_ERR_INVALID;
    *pairs = w->dev ? w->dev->p_cap : 0u;
    *contacts = w->dev ? w->dev->c_cap : 0u;
    return DYN_OK;
}

}  // extern "C"

// One step on the world's stream: the step graph, or with `taped` the taped graph that also
// snapshots the step into the tape's current slot (a segment replayed for dyn_step_backward).
static dyn_status step_once(dyn_world* w, float dt, bool taped) {
    dyn_status st = prepare_step(w, dt);
    if (st) return st;
    DeviceState* d = w->dev;
    DYN_CUDA(cudaSetDevice(w->device));
    const uint32_t slot = d->inflight_next;
    if (d->inflight_used[slot]) DYN_CUDA(cudaEventSynchronize(d->inflight[slot]));
    if ((st = widen_pair_stream(w))) return st;
    if ((st = widen_contact_stream(w))) return st;
    uint32_t parity = d->parity;
    const TapeView* tape = taped ? &d->tape.view : nullptr;
    if (w->timing) {
        for (cudaEvent_t e : d->events) cudaEventDestroy(e);
        d->events.clear();
        d->event_stage.clear();
        record_step(w, d->stream, parity, true, tape);
        DYN_CUDA(cudaGetLastError());
    } else {
        cudaGraphExec_t* exec = taped ? &d->tape.taped[parity] : &d->exec[parity];
        if (!*exec) {
            cudaGraph_t graph = nullptr;
            cudaStream_t cap = d->own_stream;
            DYN_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
            record_step(w, cap, parity, false, tape);
            cudaError_t e = cudaStreamEndCapture(cap, &graph);
            if (e != cudaSuccess) return fail(w, DYN_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            size_t nodes = 0;
            cudaGraphGetNodes(graph, nullptr, &nodes);
            std::vector<cudaGraphNode_t> list(nodes);
            cudaGraphGetNodes(graph, list.data(), &nodes);
            uint32_t kernels = 0;
            for (cudaGraphNode_t node : list) {
                cudaGraphNodeType type;
                if (cudaGraphNodeGetType(node, &type) == cudaSuccess && type == cudaGraphNodeTypeKernel) ++kernels;
            }
            if (!taped) d->graph_kernels = kernels;
            e = cudaGraphInstantiate(exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return fail(w, DYN_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        DYN_CUDA(cudaGraphLaunch(*exec, d->stream));
    }
    DYN_CUDA(cudaEventRecord(d->inflight[slot], d->stream));
    d->inflight_used[slot] = true;
    d->inflight_next = (slot + 1u) % kStepsInFlight;
    d->last_parity = parity;
    d->parity ^= 1u;
    d->stepped = true;
    return DYN_OK;
}

// ---- differentiation: checkpoints, the taped segment, the reverse graph ----
// What a step reads that an earlier step wrote: the body rows and cold body fields, the contact set
// the next step archives from (which of the two sets that is follows the parity), the counters and
// control words.
struct CheckpointPart {
    void* ptr;
    size_t bytes;
};
static std::vector<CheckpointPart> checkpoint_parts(DeviceState* d) {
    DeviceWorld& dw = d->dw;
    const size_t N = d->n_cap, C = d->c_cap;
    ContactSet& arc = d->parity == 0u ? dw.arc : dw.cur;
    return {{dw.hot, N * sizeof(BodyHot)},        {dw.prev_pos, N * sizeof(float4)}, {dw.prev_rot, N * sizeof(float4)},
            {dw.force, N * sizeof(float4)},       {dw.torque, N * sizeof(float4)},   {dw.sleep_timer, N * sizeof(float)},
            {dw.wake_flags, N * sizeof(uint32_t)}, {dw.counters, 64 * sizeof(uint32_t)}, {dw.ctl, CTL_COUNT * sizeof(uint32_t)},
            {arc.normal, C * sizeof(float4)},     {arc.rows, C * sizeof(uint4)},     {arc.mat, C * sizeof(float4)},
            {arc.ids, C * sizeof(uint4)},         {arc.ids2, C * sizeof(uint4)},     {arc.extra, C * sizeof(float4)},
            {arc.la, 4 * C * sizeof(float4)},     {arc.lb, 4 * C * sizeof(float4)},  {arc.acc, 4 * C * sizeof(float4)},
            {arc.pos, 4 * C * sizeof(float4)},
            {d->rest_ids[d->parity], (size_t)d->rest_cap * sizeof(uint4)},
            {d->rest_slots[d->parity], (size_t)d->rest_cap * sizeof(uint2)},
            // the joints' accumulated impulses and broken flags (an empty part without joints)
            {dw.jruntime, (size_t)dw.jcount * sizeof(dyn_constraint_runtime_record)}};
}
static size_t checkpoint_bytes(const std::vector<CheckpointPart>& parts) {
    size_t bytes = 0;
    for (const CheckpointPart& part : parts) bytes += (part.bytes + 255u) & ~(size_t)255u;
    return bytes;
}
static void free_checkpoint(Checkpoint* c) {
    if (c->base) cudaFree(c->base);
    c->base = nullptr;
    c->bytes = 0;
}
static dyn_status save_checkpoint(dyn_world* w, Checkpoint* c) {
    DeviceState* d = w->dev;
    const std::vector<CheckpointPart> parts = checkpoint_parts(d);
    const size_t bytes = checkpoint_bytes(parts);
    if (c->bytes != bytes) {
        free_checkpoint(c);
        DYN_CUDA(cudaMalloc(&c->base, bytes));
        c->bytes = bytes;
    }
    char* at = static_cast<char*>(c->base);
    for (const CheckpointPart& part : parts) {
        if (part.bytes) DYN_CUDA(cudaMemcpyAsync(at, part.ptr, part.bytes, cudaMemcpyDeviceToDevice, d->stream));
        at += (part.bytes + 255u) & ~(size_t)255u;
    }
    c->parity = d->parity;
    return DYN_OK;
}
static dyn_status restore_checkpoint(dyn_world* w, const Checkpoint& c) {
    DeviceState* d = w->dev;
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    d->parity = c.parity;  // before listing the parts: the archived set follows the parity
    const char* at = static_cast<const char*>(c.base);
    for (const CheckpointPart& part : checkpoint_parts(d)) {
        if (part.bytes) DYN_CUDA(cudaMemcpyAsync(part.ptr, at, part.bytes, cudaMemcpyDeviceToDevice, d->stream));
        at += (part.bytes + 255u) & ~(size_t)255u;
    }
    return DYN_OK;
}
static void free_tape_buffers(TapeHost& t) {
    for (void* p : t.tape_allocs) cudaFree(p);
    t.tape_allocs.clear();
    t.view = TapeView{};
    t.segment = -1;
}
static void free_adjoint(TapeHost& t) {
    for (void* p : t.adj_allocs) cudaFree(p);
    t.adj_allocs.clear();
    t.adj = AdjView{};
    t.grad_staging = nullptr;
    t.patch_rows = t.patch_masks = nullptr;
}
// Ends the current tape; its memory and graphs stay for the next one.
static void release_tape(DeviceState* d) {
    TapeHost& t = d->tape;
    t.checkpoint_count = 0;
    t.have_end = false;
    t.segment = -1;
    t.edit_ids.clear();
    t.edits.clear();
    t.active = false;
    t.recorded = t.reversed = 0;
}
void dyn::free_tape_memory(DeviceState* d) {
    TapeHost& t = d->tape;
    release_tape(d);
    for (auto& e : t.taped) {
        if (e) cudaGraphExecDestroy(e);
        e = nullptr;
    }
    if (t.back) cudaGraphExecDestroy(t.back);
    t.back = nullptr;
    for (Checkpoint& c : t.checkpoints) free_checkpoint(&c);
    t.checkpoints.clear();
    free_checkpoint(&t.end);
    free_tape_buffers(t);
    free_adjoint(t);
}
template <typename T>
static dyn_status tape_alloc(dyn_world* w, std::vector<void*>& list, T** out, size_t count) {
    void* p = nullptr;
    DYN_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    DYN_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(count, 1) * sizeof(T), w->dev->stream));
    list.push_back(p);
    *out = static_cast<T*>(p);
    return DYN_OK;
}
static dyn_status alloc_tape_buffers(dyn_world* w) {
    DeviceState* d = w->dev;
    TapeHost& t = d->tape;
    const dyn_step_params& p = d->params;
    if (!t.tape_allocs.empty()) {
        const TapeView& v = t.view;
        if (v.steps >= t.interval && v.substeps == p.substeps && v.iterations == p.solve_iterations &&
            v.piterations == p.position_iterations && v.n == d->n_cap && v.c == d->c_cap)
            return DYN_OK;
        DYN_CUDA(cudaStreamSynchronize(d->stream));
        free_tape_buffers(t);
        for (auto& e : t.taped) {
            if (e) cudaGraphExecDestroy(e);
            e = nullptr;
        }
        if (t.back) cudaGraphExecDestroy(t.back);
        t.back = nullptr;
    }
    TapeView& v = t.view;
    v.steps = t.interval;
    v.substeps = p.substeps;
    v.iterations = p.solve_iterations;
    v.piterations = p.position_iterations;
    v.n = d->n_cap;
    v.c = d->c_cap;
    const size_t S = v.steps, N = v.n, C = v.c, K = v.substeps;
    dyn_status st;
#define TA(field, count) if ((st = tape_alloc(w, t.tape_allocs, &v.field, (count)))) return st
    uint32_t* slot = nullptr;
    if ((st = tape_alloc(w, t.tape_allocs, &slot, 1))) return st;
    v.slot = slot;
    TA(counts, S);
    TA(rows, S * C);
    TA(normal, S * C);
    TA(mat, S * C);
    TA(ids, S * C);
    TA(extra, S * C);
    TA(la, S * 4 * C);
    TA(lb, S * 4 * C);
    TA(pos, S * 4 * C);
    TA(relay, S * 4 * C);
    TA(acc, S * K * v.iterations * 4 * C);
    TA(hot, S * (K + 1) * N);
    TA(vel, S * K * v.iterations * 2 * N);
    TA(res, S * K * v.piterations * N);
    TA(cnt, S * K * v.piterations * N);
#undef TA
    return DYN_OK;
}
static dyn_status alloc_adjoint(dyn_world* w) {
    DeviceState* d = w->dev;
    TapeHost& t = d->tape;
    if (!t.adj_allocs.empty()) return DYN_OK;
    const size_t N = d->n_cap, C = d->c_cap, K = d->k_cap;
    AdjView& a = t.adj;
    dyn_status st;
#define AA(ptr, count) if ((st = tape_alloc(w, t.adj_allocs, &(ptr), (count)))) return st
    AA(a.gx, N);
    AA(a.gq, N);
    AA(a.gv, N);
    AA(a.gw, N);
    AA(a.gv_acc, N);
    AA(a.gw_acc, N);
    AA(a.gres, N);
    AA(a.gres_acc, N);
    AA(a.gsum, N);
    AA(a.g_im, N);
    AA(a.g_scale, N);
    AA(a.g_friction, K);
    AA(a.gacc[0], 4 * C);
    AA(a.gacc[1], 4 * C);
    AA(a.acc_flip, 1);
    AA(a.g_ra, 4 * C);
    AA(a.g_rb, 4 * C);
    AA(a.g_m, 4 * C);  // float2
    AA(a.g_pt, 4 * C);
    AA(a.g_param, C);
    AA(a.t_arm_a, 4 * C);
    AA(a.t_arm_b, 4 * C);
    AA(a.t_mass, 4 * C);
    AA(a.t_tan1, C);
    AA(a.t_tan2, C);
    AA(a.t_body, C);
    AA(a.g_mu, C);
    AA(t.grad_staging, N);
    AA(t.patch_rows, N);
    AA(t.patch_masks, N);
#undef AA
    a.status = d->dw.ctl + CTL_STATUS;
    return DYN_OK;
}

// The reverse of one step (adjoint.cuh), on `s`.
static void record_backward_step(dyn_world* w, cudaStream_t s) {
    DeviceState* d = w->dev;
    const TapeView& t = d->tape.view;
    const AdjView& a = d->tape.adj;
    const dyn_step_params p = d->params;
    const uint32_t n = std::max(d->dw.n, 1u);
    const uint32_t C = d->c_cap;
    const uint32_t rows_grid = blocks_for(d, n, 256), contact_grid = blocks_for(d, C, 128);
    const uint32_t quad_grid = blocks_for(d, 4 * C, 128);  // a quad of lanes per contact block
    k_adj_begin<<<1, 32, 0, s>>>(t, a);
    k_adj_clear<<<blocks_for(d, std::max(4 * C, n), 256), 256, 0, s>>>(t, a, n);
    for (int32_t k = (int32_t)p.substeps - 1; k >= 0; --k) {
        k_adj_terms<<<contact_grid, 128, 0, s>>>(t, a, (uint32_t)k);
        const uint32_t P = p.position_iterations;
        if (P > 0) {
            k_adj_prow<<<rows_grid, 256, 0, s>>>(t, a, n, (uint32_t)k, P - 1, false, true);
            for (int32_t it = (int32_t)P - 1; it >= 0; --it) {
                k_adj_pcontact<<<contact_grid, 128, 0, s>>>(t, a, p, (uint32_t)k, (uint32_t)it);
                k_adj_prow<<<rows_grid, 256, 0, s>>>(t, a, n, (uint32_t)k, it > 0 ? (uint32_t)(it - 1) : 0u, true, it > 0);
            }
        }
        k_adj_advance<<<rows_grid, 256, 0, s>>>(t, a, n, p, (uint32_t)k);
        for (int32_t it = (int32_t)p.solve_iterations - 1; it >= 0; --it) {
            k_adj_solve<<<quad_grid, 128, 0, s>>>(t, a, p, (uint32_t)k, (uint32_t)it);
            k_adj_vmerge<<<rows_grid, 256, 0, s>>>(a, n);
        }
        if (k == 0) k_adj_warm<<<contact_grid, 128, 0, s>>>(t, a);
        k_adj_prepare<<<contact_grid, 128, 0, s>>>(t, a, (uint32_t)k);
        k_adj_integrate<<<rows_grid, 256, 0, s>>>(d->dw, t, a, p, (uint32_t)k);
    }
    k_adj_start<<<contact_grid, 128, 0, s>>>(d->dw, t, a, p);
    k_adj_end<<<1, 32, 0, s>>>(a);
}

// Steps the recorded steps of segment `seg` again from its checkpoint, taped.
static dyn_status materialize_segment(dyn_world* w, int32_t seg) {
    DeviceState* d = w->dev;
    TapeHost& t = d->tape;
    if (t.segment == seg) return DYN_OK;
    dyn_status st = alloc_tape_buffers(w);
    if (st) return st;
    if ((st = restore_checkpoint(w, t.checkpoints[(size_t)seg]))) return st;
    DYN_CUDA(cudaMemsetAsync(t.view.slot, 0, sizeof(uint32_t), d->stream));
    const uint32_t first = (uint32_t)seg * t.interval;
    const uint32_t last = std::min(t.recorded, first + t.interval);
    for (uint32_t j = first; j < last; ++j) {
        w->edit_ids = t.edit_ids[j];
        w->edits = t.edits[j];
        if ((st = step_once(w, t.dt, true))) return st;
    }
    t.segment = seg;
    return DYN_OK;
}

// The rows and PATCH masks of recorded step j's edits, onto the device; returns how many.
static dyn_status upload_patches(dyn_world* w, uint32_t j, uint32_t* count) {
    DeviceState* d = w->dev;
    TapeHost& t = d->tape;
    std::vector<uint32_t> rows, masks;
    for (size_t e = 0; e < t.edits[j].size(); ++e) {
        const uint32_t id = t.edit_ids[j][e];
        const uint32_t row = id < w->row_of_id.size() ? w->row_of_id[id] : DYN_NO_BODY;
        if (row == DYN_NO_BODY || row >= d->dw.n) continue;
        rows.push_back(row);
        masks.push_back(t.edits[j][e].mask);
    }
    *count = (uint32_t)rows.size();
    if (rows.empty()) return DYN_OK;
    DYN_CUDA(cudaMemcpyAsync(t.patch_rows, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice, d->stream));
    DYN_CUDA(cudaMemcpyAsync(t.patch_masks, masks.data(), masks.size() * 4, cudaMemcpyHostToDevice, d->stream));
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    return DYN_OK;
}

static dyn_status backward_steps(dyn_world* w, const dyn_body_grad* grad_in, dyn_body_grad* grad_out, uint32_t n,
                                 uint32_t steps) {
    if (!w || !grad_in || !grad_out) return DYN_ERR_INVALID;
    DeviceState* d = w->dev;
    if (!d || !d->tape.active) return fail(w, DYN_ERR_INVALID, "dyn_step_backward: no tape is recording (dyn_tape_begin)");
    TapeHost& t = d->tape;
    if (n != d->dw.n) return fail(w, DYN_ERR_INVALID, "dyn_step_backward: n differs from the world's body rows");
    if (steps == 0 || steps > t.recorded - t.reversed)
        return fail(w, DYN_ERR_INVALID, "dyn_step_backward: fewer recorded steps are left to reverse");
    DYN_CUDA(cudaSetDevice(w->device));
    dyn_status st;
    if (!t.have_end) {
        DYN_CUDA(cudaStreamSynchronize(d->stream));
        if ((st = save_checkpoint(w, &t.end))) return st;
        t.have_end = true;
    }
    if ((st = alloc_adjoint(w))) return st;
    DYN_CUDA(cudaMemcpyAsync(t.grad_staging, grad_in, (size_t)n * sizeof(dyn_body_grad), cudaMemcpyHostToDevice, d->stream));
    k_grad_unpack<<<blocks_for(d, n, 256), 256, 0, d->stream>>>(t.adj, t.grad_staging, n);
    DYN_CUDA(cudaGetLastError());
    for (uint32_t k = 0; k < steps; ++k) {
        const uint32_t step = t.recorded - t.reversed - 1u;
        if (k > 0) {
            // the step after this one replaced some fields by edits: no gradient reaches past them
            uint32_t m = 0;
            if ((st = upload_patches(w, step + 1u, &m))) return st;
            if (m) k_adj_patch<<<blocks_for(d, m, 256), 256, 0, d->stream>>>(t.adj, t.patch_rows, t.patch_masks, m);
        }
        const int32_t seg = (int32_t)(step / t.interval);
        if ((st = materialize_segment(w, seg))) return st;
        if (!t.back) {
            alloc_tape_buffers(w);
            cudaGraph_t graph = nullptr;
            cudaStream_t cap = d->own_stream;
            DYN_CUDA(cudaStreamSynchronize(d->stream));
            DYN_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
            record_backward_step(w, cap);
            cudaError_t e = cudaStreamEndCapture(cap, &graph);
            if (e != cudaSuccess) return fail(w, DYN_ERR_CUDA, std::string("backward graph capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&t.back, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return fail(w, DYN_ERR_CUDA, std::string("backward graph instantiate: ") + cudaGetErrorString(e));
        }
        DYN_CUDA(cudaGraphLaunch(t.back, d->stream));
        t.reversed += 1u;
        if (step % t.interval == 0u) t.segment = -1;  // the segment's slots are all consumed
    }
    k_grad_pack<<<blocks_for(d, n, 256), 256, 0, d->stream>>>(t.adj, t.grad_staging, n);
    DYN_CUDA(cudaGetLastError());
    DYN_CUDA(cudaMemcpyAsync(grad_out, t.grad_staging, (size_t)n * sizeof(dyn_body_grad), cudaMemcpyDeviceToHost, d->stream));
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    return DYN_OK;
}

extern "C" {

DYN_API dyn_status dyn_step(dyn_world* w, float dt) {
    if (!w) return DYN_ERR_INVALID;
    DeviceState* d = w->dev;
    const bool recording = d && d->tape.active;
    if (recording) {
        TapeHost& t = d->tape;
        if (t.reversed > 0) return fail(w, DYN_ERR_INVALID, "dyn_step: the tape is being reversed (dyn_tape_end first)");
        if (t.recorded > 0 && dt != t.dt) return fail(w, DYN_ERR_INVALID, "dyn_step: every recorded step takes one timestep");
        for (const dyn_body_edit_record& e : w->edits) {
            if (e.kind != DYN_EDIT_PATCH) return fail(w, DYN_ERR_INVALID, "dyn_step: only PATCH edits while recording");
        }
        if (w->rows_dirty && !w->raw_rows) return fail(w, DYN_ERR_INVALID, "dyn_step: the scene changed while recording");
        if (t.recorded > 0 && t.recorded % t.interval == 0u) {
            if (t.checkpoints.size() <= t.checkpoint_count) t.checkpoints.emplace_back();
            dyn_status st = save_checkpoint(w, &t.checkpoints[t.checkpoint_count]);
            if (st) return st;
            t.checkpoint_count += 1;
        }
        t.edit_ids.push_back(w->edit_ids);
        t.edits.push_back(w->edits);
        t.dt = dt;
    }
    dyn_status st = step_once(w, dt, false);
    if (st) return st;
    if (recording) w->dev->tape.recorded += 1u;
    w->steps_taken += 1;
    if (w->observer.active) return observe_after_step(w);
    return DYN_OK;
}

DYN_API dyn_status dyn_tape_begin(dyn_world* w, uint32_t checkpoint_interval) {
    if (!w || checkpoint_interval == 0) return fail(w, DYN_ERR_INVALID, "dyn_tape_begin: the checkpoint interval must be > 0");
    if (std::isfinite(w->config.sleep_time)) return fail(w, DYN_ERR_INVALID, "dyn_tape_begin: sleeping must be off (sleep_time = inf)");
    if (!w->joint_descs.empty()) return fail(w, DYN_ERR_INVALID, "dyn_tape_begin: constraints are not differentiated");
    if (w->solver_guard) return fail(w, DYN_ERR_INVALID, "dyn_tape_begin: the adjoint differentiates the reference's solver (no guard)");
    rebuild_rows(w);
    if (world_has_ccd(w)) return fail(w, DYN_ERR_INVALID, "dyn_tape_begin: continuous collision is not differentiated");
    for (uint32_t i = 0; i < w->dynamic_count && i < w->descs.size(); ++i) {
        const float* ii = w->descs[i].inverse_inertia;
        if (w->descs[i].inverse_mass > 0.0f && !(ii[1] == 0.0f && ii[2] == 0.0f && ii[4] == 0.0f && ii[0] == ii[3] && ii[3] == ii[5]))
            return fail(w, DYN_ERR_INVALID, "dyn_tape_begin: a dynamic body's inverse inertia is not isotropic");
    }
    bool fresh = !w->dev || !w->dev->uploaded || (w->rows_dirty && !w->raw_rows) || w->scene_dirty;
    if (fresh) {
        dyn_status st = upload_scene(w);
        if (st) return st;
    }
    DeviceState* d = w->dev;
    DYN_CUDA(cudaSetDevice(w->device));
    release_tape(d);
    TapeHost& t = d->tape;
    t.interval = checkpoint_interval;
    t.active = true;
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    if (t.checkpoints.empty()) t.checkpoints.emplace_back();
    dyn_status st = save_checkpoint(w, &t.checkpoints[0]);
    if (st) {
        release_tape(d);
        return st;
    }
    t.checkpoint_count = 1;
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    return DYN_OK;
}

DYN_API dyn_status dyn_tape_end(dyn_world* w) {
    if (!w) return DYN_ERR_INVALID;
    DeviceState* d = w->dev;
    if (!d || !d->tape.active) return DYN_OK;
    DYN_CUDA(cudaSetDevice(w->device));
    if (d->tape.have_end) {
        dyn_status st = restore_checkpoint(w, d->tape.end);
        if (st) return st;
    }
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    release_tape(d);
    return DYN_OK;
}

DYN_API dyn_status dyn_tape_steps(const dyn_world* w, uint32_t* recorded, uint32_t* reversed) {
    if (!w) return DYN_ERR_INVALID;
    const bool on = w->dev && w->dev->tape.active;
    if (recorded) *recorded = on ? w->dev->tape.recorded : 0u;
    if (reversed) *reversed = on ? w->dev->tape.reversed : 0u;
    return DYN_OK;
}

DYN_API dyn_status dyn_step_backward(dyn_world* w, const dyn_body_grad* grad_in, dyn_body_grad* grad_out, uint32_t n) {
    return backward_steps(w, grad_in, grad_out, n, 1u);
}

DYN_API dyn_status dyn_backward(dyn_world* w, const dyn_body_grad* grad_in, dyn_body_grad* grad_out, uint32_t n, uint32_t steps) {
    return backward_steps(w, grad_in, grad_out, n, steps);
}

DYN_API dyn_status dyn_set_mass_properties(dyn_world* w, const float* inverse_mass, const float* inverse_inertia, uint32_t n) {
    if (!w || !inverse_mass || !inverse_inertia) return fail(w, DYN_ERR_INVALID, "dyn_set_mass_properties: null argument");
    if (w->dev && w->dev->tape.active) return fail(w, DYN_ERR_INVALID, "dyn_set_mass_properties: a tape is recording");
    rebuild_rows(w);
    if (n != w->descs.size()) return fail(w, DYN_ERR_INVALID, "dyn_set_mass_properties: n differs from the body rows");
    for (uint32_t r = 0; r < n; ++r) {
        const bool dynamic = r < w->dynamic_count;
        if (!std::isfinite(inverse_mass[r]) || (dynamic != (inverse_mass[r] > 0.0f)))
            return fail(w, DYN_ERR_INVALID, "dyn_set_mass_properties: a row would change between dynamic and static");
        for (int k = 0; k < 6; ++k) {
            if (!std::isfinite(inverse_inertia[6 * (size_t)r + k]))
                return fail(w, DYN_ERR_INVALID, "dyn_set_mass_properties: inverse inertia must be finite");
        }
    }
    std::vector<uint32_t> id_of_row(n, DYN_NO_BODY);
    for (uint32_t id = 0; id < w->row_of_id.size(); ++id) {
        if (w->row_of_id[id] < n) id_of_row[w->row_of_id[id]] = id;
    }
    std::vector<float> inertia(6 * (size_t)n, 0.0f);
    for (uint32_t r = 0; r < n; ++r) {
        const float* t = inverse_inertia + 6 * (size_t)r;
        // the inertia is the inverse of the symmetric tensor (xx, xy, xz, yy, yz, zz); zero stays zero
        const double a = t[0], b = t[1], c = t[2], d = t[3], e = t[4], f = t[5];
        const double c00 = d * f - e * e, c01 = c * e - b * f, c02 = b * e - c * d;
        const double det = a * c00 + b * c01 + c * c02;
        float* I = &inertia[6 * (size_t)r];
        if (det != 0.0) {
            I[0] = (float)(c00 / det);
            I[1] = (float)(c01 / det);
            I[2] = (float)(c02 / det);
            I[3] = (float)((a * f - c * c) / det);
            I[4] = (float)((b * c - a * e) / det);
            I[5] = (float)((a * d - b * b) / det);
        }
        dyn_body_descriptor_record& rec = w->descs[r];
        rec.inverse_mass = inverse_mass[r];
        for (int k = 0; k < 6; ++k) {
            rec.inverse_inertia[k] = t[k];
            rec.inertia[k] = I[k];
        }
        if (!w->raw_rows && id_of_row[r] < w->spawn_descs.size()) w->spawn_descs[id_of_row[r]] = rec;
    }
    DeviceState* d = w->dev;
    if (d && d->uploaded) {
        DYN_CUDA(cudaSetDevice(w->device));
        float *dim = nullptr, *dii = nullptr, *din = nullptr;
        DYN_CUDA(cudaMalloc(&dim, (size_t)n * 4));
        DYN_CUDA(cudaMalloc(&dii, (size_t)n * 24));
        DYN_CUDA(cudaMalloc(&din, (size_t)n * 24));
        cudaMemcpyAsync(dim, inverse_mass, (size_t)n * 4, cudaMemcpyHostToDevice, d->stream);
        cudaMemcpyAsync(dii, inverse_inertia, (size_t)n * 24, cudaMemcpyHostToDevice, d->stream);
        cudaMemcpyAsync(din, inertia.data(), (size_t)n * 24, cudaMemcpyHostToDevice, d->stream);
        k_set_mass<<<blocks_for(d, n, 256), 256, 0, d->stream>>>(d->dw, dim, dii, din, n);
        cudaError_t e = cudaStreamSynchronize(d->stream);
        cudaFree(dim);
        cudaFree(dii);
        cudaFree(din);
        if (e != cudaSuccess) return fail(w, DYN_ERR_CUDA, std::string("dyn_set_mass_properties: ") + cudaGetErrorString(e));
    }
    return DYN_OK;
}

DYN_API dyn_status dyn_set_friction(dyn_world* w, const float* friction, uint32_t k) {
    if (!w || !friction) return fail(w, DYN_ERR_INVALID, "dyn_set_friction: null argument");
    if (w->dev && w->dev->tape.active) return fail(w, DYN_ERR_INVALID, "dyn_set_friction: a tape is recording");
    rebuild_rows(w);
    if (k != w->colliders.size()) return fail(w, DYN_ERR_INVALID, "dyn_set_friction: k differs from the colliders");
    for (uint32_t c = 0; c < k; ++c) {
        if (!(friction[c] >= 0.0f) || !std::isfinite(friction[c])) return fail(w, DYN_ERR_INVALID, "dyn_set_friction: friction must be >= 0");
    }
    for (uint32_t c = 0; c < k; ++c) w->colliders[c].friction = friction[c];
    if (!w->raw_rows) {
        uint32_t c = 0;
        for (size_t i = 0; i < w->spawn_owner.size() && c < k; ++i) {
            if (w->removed.size() > w->spawn_owner[i] && w->removed[w->spawn_owner[i]]) continue;
            w->spawn_colliders[i].friction = friction[c++];
        }
    }
    DeviceState* d = w->dev;
    if (d && d->uploaded) {
        DYN_CUDA(cudaSetDevice(w->device));
        float* df = nullptr;
        DYN_CUDA(cudaMalloc(&df, (size_t)k * 4));
        cudaMemcpyAsync(df, friction, (size_t)k * 4, cudaMemcpyHostToDevice, d->stream);
        k_set_friction<<<blocks_for(d, k, 256), 256, 0, d->stream>>>(d->dw, df, k);
        cudaError_t e = cudaStreamSynchronize(d->stream);
        cudaFree(df);
        if (e != cudaSuccess) return fail(w, DYN_ERR_CUDA, std::string("dyn_set_friction: ") + cudaGetErrorString(e));
    }
    return DYN_OK;
}

DYN_API dyn_status dyn_param_grads(dyn_world* w, float* inverse_mass, float* inertia_scale, uint32_t n, float* friction,
                                   uint32_t k) {
    if (!w) return DYN_ERR_INVALID;
    DeviceState* d = w->dev;
    const bool have = d && d->tape.active && !d->tape.adj_allocs.empty();
    if (have) DYN_CUDA(cudaStreamSynchronize(d->stream));
    const uint32_t rows = have ? d->dw.n : 0u, colliders = have ? d->dw.k : 0u;
    if (inverse_mass) {
        std::memset(inverse_mass, 0, (size_t)n * 4);
        if (have) DYN_CUDA(cudaMemcpy(inverse_mass, d->tape.adj.g_im, (size_t)std::min(n, rows) * 4, cudaMemcpyDeviceToHost));
    }
    if (inertia_scale) {
        std::memset(inertia_scale, 0, (size_t)n * 4);
        if (have) DYN_CUDA(cudaMemcpy(inertia_scale, d->tape.adj.g_scale, (size_t)std::min(n, rows) * 4, cudaMemcpyDeviceToHost));
    }
    if (friction) {
        std::memset(friction, 0, (size_t)k * 4);
        if (have) DYN_CUDA(cudaMemcpy(friction, d->tape.adj.g_friction, (size_t)std::min(k, colliders) * 4, cudaMemcpyDeviceToHost));
    }
    return DYN_OK;
}

DYN_API dyn_status dyn_observe_bodies(dyn_world* w, const uint32_t* body_ids, uint32_t n) {
    if (!w || (n && !body_ids)) return fail(w, DYN_ERR_INVALID, "dyn_observe_bodies: null argument");
    Observer& o = w->observer;
    if (!body_ids) {
        o.all = true;
        o.ids.clear();
    } else {
        const uint32_t ids = (uint32_t)std::max(w->spawn_states.size(), w->row_of_id.size());
        for (uint32_t i = 0; i < n; ++i) {
            if (body_ids[i] >= ids) return fail(w, DYN_ERR_INVALID, "dyn_observe_bodies: unknown body id");
        }
        if (o.all) o.ids.clear();
        o.all = false;
        o.ids.insert(o.ids.end(), body_ids, body_ids + n);
        std::sort(o.ids.begin(), o.ids.end());
        o.ids.erase(std::unique(o.ids.begin(), o.ids.end()), o.ids.end());
        o.ids_dirty = true;
    }
    o.active = true;
    return DYN_OK;
}

DYN_API dyn_status dyn_stop_observing(dyn_world* w) {
    if (!w) return DYN_ERR_INVALID;
    w->observer.active = false;
    w->observer.all = false;
    w->observer.ids.clear();
    return DYN_OK;
}

DYN_API dyn_status dyn_poll(dyn_world* w) {
    if (!w) return DYN_ERR_INVALID;
    observer_poll(w);
    return DYN_OK;
}

DYN_API dyn_status dyn_try_state(dyn_world* w, uint32_t body_id, dyn_body_state_record* out, uint64_t* step) {
    if (!w || !out) return DYN_ERR_INVALID;
    observer_poll(w);
    Observer& o = w->observer;
    if (o.latest < 0) return DYN_NOT_READY;
    ObservationSlot& s = o.slots[o.latest];
    const dyn_body_state_record* records = static_cast<const dyn_body_state_record*>(s.states);
    if (s.index_of_id.empty() && s.count > 0) {
        uint32_t top = 0;
        for (uint32_t i = 0; i < s.count; ++i) {
            if (records[i].body_id != DYN_NO_BODY) top = std::max(top, records[i].body_id);
        }
        s.index_of_id.assign((size_t)top + 1, DYN_NO_BODY);
        for (uint32_t i = 0; i < s.count; ++i) {
            if (records[i].body_id != DYN_NO_BODY) s.index_of_id[records[i].body_id] = i;
        }
    }
    if (body_id >= s.index_of_id.size() || s.index_of_id[body_id] == DYN_NO_BODY)
        return fail(w, DYN_ERR_INVALID, "dyn_try_state: the body is not in the latest observation");
    *out = records[s.index_of_id[body_id]];
    if (step) *step = s.step;
    return DYN_OK;
}

DYN_API dyn_status dyn_try_counters(dyn_world* w, uint32_t* out, uint32_t n, uint64_t* step) {
    if (!w || !out) return DYN_ERR_INVALID;
    observer_poll(w);
    Observer& o = w->observer;
    if (o.latest < 0) return DYN_NOT_READY;
    const ObservationSlot& s = o.slots[o.latest];
    std::memcpy(out, s.counters, (size_t)std::min<uint32_t>(n, DYN_COUNTER_DEVICE_COUNT) * 4);
    if (step) *step = s.step;
    return DYN_OK;
}

DYN_API dyn_status dyn_sync(dyn_world* w) {
    if (!w) return DYN_ERR_INVALID;
    if (!w->dev) return DYN_OK;
    DYN_CUDA(cudaStreamSynchronize(w->dev->stream));
    uint32_t status = 0;
    DYN_CUDA(cudaMemcpy(&status, w->dev->dw.ctl + CTL_STATUS, 4, cudaMemcpyDeviceToHost));
    if (status) return fail(w, DYN_ERR_DEVICE_STATUS, "device status word " + std::to_string(status));
    return DYN_OK;
}

DYN_API dyn_status dyn_read_constraints(dyn_world* w, dyn_constraint_runtime_record* out, uint32_t m) {
    if (!w || (m && !out)) return fail(w, DYN_ERR_INVALID, "dyn_read_constraints: null argument");
    if (m != w->joint_descs.size()) return fail(w, DYN_ERR_INVALID, "dyn_read_constraints: count differs from the constraints");
    DeviceState* d = w->dev;
    if (d && d->uploaded && !w->joints_dirty && d->dw.jcount == m && m) {
        DYN_CUDA(cudaStreamSynchronize(d->stream));
        DYN_CUDA(cudaMemcpy(out, d->dw.jruntime, (size_t)m * sizeof(*out), cudaMemcpyDeviceToHost));
        return DYN_OK;
    }
    if (m) std::memcpy(out, w->joint_runtime.data(), (size_t)m * sizeof(*out));
    return DYN_OK;
}

DYN_API dyn_status dyn_device_status(dyn_world* w, uint32_t* status) {
    if (!w || !status) return DYN_ERR_INVALID;
    *status = 0;
    if (!w->dev) return DYN_OK;
    DYN_CUDA(cudaStreamSynchronize(w->dev->stream));
    DYN_CUDA(cudaMemcpy(status, w->dev->dw.ctl + CTL_STATUS, 4, cudaMemcpyDeviceToHost));
    return DYN_OK;
}

DYN_API dyn_status dyn_download_states(dyn_world* w, dyn_body_state_record* out, uint32_t n) {
    if (!w || !out) return DYN_ERR_INVALID;
    rebuild_rows(w);
    if (!w->dev || !w->dev->uploaded) {
        if (n < w->states.size()) return DYN_ERR_INVALID;
        std::memcpy(out, w->states.data(), w->states.size() * sizeof(*out));
        return DYN_OK;
    }
    DeviceState* d = w->dev;
    uint32_t rows = d->dw.n;
    if (n < rows) return fail(w, DYN_ERR_INVALID, "dyn_download_states: buffer too small");
    k_pack_states<<<blocks_for(d, std::max(rows, 1u), 256), 256, 0, d->stream>>>(d->dw, d->staging, rows);
    DYN_CUDA(cudaGetLastError());
    DYN_CUDA(cudaMemcpyAsync(out, d->staging, (size_t)rows * sizeof(dyn_body_state_record), cudaMemcpyDeviceToHost,
                             d->stream));
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    return DYN_OK;
}

DYN_API dyn_status dyn_read_state(dyn_world* w, uint32_t body_id, dyn_body_state_record* out) {
    if (!w || !out) return DYN_ERR_INVALID;
    rebuild_rows(w);
    if (body_id >= w->row_of_id.size() || w->row_of_id[body_id] == DYN_NO_BODY) return fail(w, DYN_ERR_INVALID, "unknown body id");
    uint32_t row = w->row_of_id[body_id];
    if (!w->dev || !w->dev->uploaded) {
        *out = w->states[row];
        return DYN_OK;
    }
    std::vector<dyn_body_state_record> states;
    dyn_status st = download_states(w, &states);
    if (st) return st;
    *out = states[row];
    return DYN_OK;
}

DYN_API dyn_status dyn_read_counters(dyn_world* w, uint32_t* out, uint32_t n) {
    if (!w || !out) return DYN_ERR_INVALID;
    uint32_t m = std::min<uint32_t>(n, DYN_COUNTER_DEVICE_COUNT);
    if (!w->dev) {
        std::memset(out, 0, m * 4);
        return DYN_OK;
    }
    DYN_CUDA(cudaStreamSynchronize(w->dev->stream));
    DYN_CUDA(cudaMemcpy(out, w->dev->dw.counters, m * 4, cudaMemcpyDeviceToHost));
    return DYN_OK;
}

DYN_API dyn_status dyn_debug_aabbs(dyn_world* w, dyn_aabb_record* out, uint32_t cap, uint32_t* count) {
    if (!w || !w->dev) return DYN_ERR_INVALID;
    DeviceWorld& dw = w->dev->dw;
    if (count) *count = dw.k;
    if (!out) return DYN_OK;
    uint32_t m = std::min(cap, dw.k);
    DYN_CUDA(cudaStreamSynchronize(w->dev->stream));
    DYN_CUDA(cudaMemcpy(out, dw.aabb, m * sizeof(dyn_aabb_record), cudaMemcpyDeviceToHost));
    return DYN_OK;
}

DYN_API dyn_status dyn_debug_entries(dyn_world* w, uint32_t* keys, uint32_t* infos, uint32_t cap, uint32_t* count) {
    if (!w || !w->dev) return DYN_ERR_INVALID;
    DeviceWorld& dw = w->dev->dw;
    DYN_CUDA(cudaStreamSynchronize(w->dev->stream));
    uint32_t e = 0;
    DYN_CUDA(cudaMemcpy(&e, dw.ctl + CTL_ENTRIES, 4, cudaMemcpyDeviceToHost));
    e = std::min(e, dw.e_cap);
    if (count) *count = e;
    if (!keys) return DYN_OK;
    uint32_t m = std::min(cap, e);
    std::vector<uint32_t> order(m);
    std::vector<float4> ent(2 * (size_t)dw.e_cap);  // slots are the colliders' windows, up to e_cap
    DYN_CUDA(cudaMemcpy(keys, dw.ekey, m * 4, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(order.data(), dw.eval, m * 4, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(ent.data(), dw.entries, ent.size() * sizeof(float4), cudaMemcpyDeviceToHost));
    if (infos) {
        for (uint32_t i = 0; i < m; ++i) {
            float f = ent[2 * (size_t)order[i] + 1].w;
            std::memcpy(&infos[i], &f, 4);
        }
    }
    return DYN_OK;
}

DYN_API dyn_status dyn_debug_pairs(dyn_world* w, uint32_t* major, uint32_t* minor, uint32_t cap, uint32_t* count) {
    if (!w || !w->dev) return DYN_ERR_INVALID;
    DeviceWorld& dw = w->dev->dw;
    DYN_CUDA(cudaStreamSynchronize(w->dev->stream));
    uint32_t p = 0;
    DYN_CUDA(cudaMemcpy(&p, dw.counters + DYN_COUNTER_PAIRS, 4, cudaMemcpyDeviceToHost));
    p = std::min(p, dw.p_cap);
    if (count) *count = p;
    if (!major) return DYN_OK;
    // the device keeps the pairs in emission order; the readback sorts them (the reference's order)
    std::vector<uint32_t> maj(p), mnr(p);
    DYN_CUDA(cudaMemcpy(maj.data(), dw.pmaj, (size_t)p * 4, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(mnr.data(), dw.pmin, (size_t)p * 4, cudaMemcpyDeviceToHost));
    std::vector<uint64_t> keys(p);
    for (uint32_t i = 0; i < p; ++i) keys[i] = ((uint64_t)maj[i] << 32) | mnr[i];
    std::sort(keys.begin(), keys.end());
    uint32_t m = std::min(cap, p);
    for (uint32_t i = 0; i < m; ++i) {
        major[i] = (uint32_t)(keys[i] >> 32);
        minor[i] = (uint32_t)keys[i];
    }
    return DYN_OK;
}

DYN_API dyn_status dyn_debug_contacts(dyn_world* w, dyn_contact_record* out, uint32_t cap, uint32_t* count) {
    if (!w || !w->dev) return DYN_ERR_INVALID;
    DeviceState* d = w->dev;
    DeviceWorld dw = d->dw;
    if (d->last_parity) std::swap(dw.cur, dw.arc);
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    uint32_t c = 0;
    DYN_CUDA(cudaMemcpy(&c, dw.ctl + CTL_CONTACTS, 4, cudaMemcpyDeviceToHost));
    if (!d->stepped) c = 0;
    if (count) *count = c;
    if (!out) return DYN_OK;
    // the device keeps the contacts in the order the narrowphase appended them; the readback sorts
    // them by collider pair (the reference's compacted order)
    uint32_t m = c;
    uint32_t C = dw.c_cap;
    std::vector<float4> normal(m), mat(m), extra(m), la(4 * (size_t)C), lb(4 * (size_t)C), acc(4 * (size_t)C), pos(4 * (size_t)C);
    std::vector<uint4> rows(m), ids(m), ids2(m);
    std::vector<dyn_contact_record> all(m);
    DYN_CUDA(cudaMemcpy(normal.data(), dw.cur.normal, m * 16, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(mat.data(), dw.cur.mat, m * 16, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(extra.data(), dw.cur.extra, m * 16, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(rows.data(), dw.cur.rows, m * 16, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(ids.data(), dw.cur.ids, m * 16, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(ids2.data(), dw.cur.ids2, m * 16, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(la.data(), dw.cur.la, 4 * (size_t)C * 16, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(lb.data(), dw.cur.lb, 4 * (size_t)C * 16, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(acc.data(), dw.cur.acc, 4 * (size_t)C * 16, cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(pos.data(), dw.cur.pos, 4 * (size_t)C * 16, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < m; ++i) {
        dyn_contact_record& r = all[i];
        std::memset(&r, 0, sizeof(r));
        r.a = ids[i].x;
        r.b = ids[i].y;
        r.point_count = rows[i].z & 0xFFu;
        r.sensor = (rows[i].z >> 8) & 0xFFu;
        r.first_body_id = ids[i].z;
        r.second_body_id = ids[i].w;
        r.first_generation = ids2[i].x;
        r.second_generation = ids2[i].y;
        r.normal[0] = normal[i].x;
        r.normal[1] = normal[i].y;
        r.normal[2] = normal[i].z;
        r.events = rows[i].w;
        r.surface = ids2[i].z;
        r.triangle = ids2[i].w;
        r.friction = normal[i].w;
        r.restitution = extra[i].x;
        r.rolling_friction = mat[i].x;
        r.spin_friction = mat[i].y;
        r.carried_normal = extra[i].y;
        r.carried_tangent = extra[i].z;
        r.relaxation = mat[i].z;
        r.damping_ratio = mat[i].w;
        for (uint32_t p = 0; p < r.point_count && p < 4; ++p) {
            size_t o = (size_t)p * C + i;
            dyn_manifold_point_record& q = r.points[p];
            q.position[0] = pos[o].x;
            q.position[1] = pos[o].y;
            q.position[2] = pos[o].z;
            q.depth = la[o].w;
            q.local_a[0] = la[o].x;
            q.local_a[1] = la[o].y;
            q.local_a[2] = la[o].z;
            q.local_b[0] = lb[o].x;
            q.local_b[1] = lb[o].y;
            q.local_b[2] = lb[o].z;
            q.accumulated_normal = acc[o].x;
            q.accumulated_tangent_1 = acc[o].y;
            q.accumulated_tangent_2 = acc[o].z;
            std::memcpy(&q.feature, &acc[o].w, 4);
        }
    }
    std::sort(all.begin(), all.end(), [](const dyn_contact_record& x, const dyn_contact_record& y) {
        return x.a < y.a || (x.a == y.a && x.b < y.b);
    });
    std::memcpy(out, all.data(), (size_t)std::min(cap, c) * sizeof(dyn_contact_record));
    return DYN_OK;
}

DYN_API dyn_status dyn_debug_islands(dyn_world* w, uint32_t* out, uint32_t cap, uint32_t* count) {
    if (!w || !w->dev) return DYN_ERR_INVALID;
    DeviceWorld& dw = w->dev->dw;
    if (count) *count = dw.nd;
    if (!out) return DYN_OK;
    DYN_CUDA(cudaStreamSynchronize(w->dev->stream));
    DYN_CUDA(cudaMemcpy(out, dw.parents, std::min(cap, dw.nd) * 4, cudaMemcpyDeviceToHost));
    return DYN_OK;
}

// Validates one query as the reference's constructors assert (crates/dynamis-abi/src/query.rs:103-181,
// crates/dynamis-world/src/query.rs:82-125): finite vectors, a non-zero direction, positive lengths,
// a convex probe shape.
static bool query_valid(const dyn_world* w, const dyn_query_record& q) {
    auto finite3 = [](const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); };
    if (q.kind > DYN_QUERY_CONVEX || q.max_hits == 0u || !finite3(q.origin)) return false;
    const bool directed = q.kind == DYN_QUERY_RAY || q.kind == DYN_QUERY_SWEEP;
    if (directed && (!finite3(q.direction) || (q.direction[0] == 0.0f && q.direction[1] == 0.0f && q.direction[2] == 0.0f)))
        return false;
    if (directed && !(q.extent > 0.0f && std::isfinite(q.extent))) return false;
    if (q.kind == DYN_QUERY_SPHERE && !(q.radius > 0.0f && q.extent > 0.0f)) return false;
    if (q.kind == DYN_QUERY_CUBOID && !(q.half_extents[0] > 0.0f && q.half_extents[1] > 0.0f && q.half_extents[2] > 0.0f))
        return false;
    // QueryRecord::cuboid, ::sphere and ::point leave the orientation zero (query.rs:115-144); the
    // shaped probes of overlap and sweep queries carry a unit one (query.rs:146-181)
    if (q.kind == DYN_QUERY_CONVEX || q.kind == DYN_QUERY_SWEEP) {
        const uint32_t k = q.shape_kind;
        if (!(k == DYN_SHAPE_SPHERE || k == DYN_SHAPE_CUBOID || k == DYN_SHAPE_CAPSULE || k == DYN_SHAPE_CYLINDER ||
              k == DYN_SHAPE_HULL))
            return false;
        if (k == DYN_SHAPE_HULL && q.source >= w->hulls.size()) return false;
        const float* o = q.orientation;
        const float norm = o[0] * o[0] + o[1] * o[1] + o[2] * o[2] + o[3] * o[3];
        if (!(std::fabs(norm - 1.0f) <= 1e-3f)) return false;
    }
    return true;
}

// World::ray_query ... sweep_query, resolve_queries and query_hits (crates/dynamis-world/src/query.rs:50-175,
// the Query pass of crates/dynamis-scene/src/passes.rs:15-39) as one call.
DYN_API dyn_status dyn_query(dyn_world* w, dyn_query_record* queries, uint32_t n, dyn_query_hit_record* hits, uint32_t hit_capacity) {
    if (!w || (n && (!queries || !hits))) return fail(w, DYN_ERR_INVALID, "dyn_query: null argument");
    if (n == 0) return DYN_OK;
    rebuild_rows(w);
    for (uint32_t b : w->body_world) {
        if (b != 0u) return fail(w, DYN_ERR_INVALID, "dyn_query: a world of batched sub-worlds takes no scene queries");
    }
    uint64_t base = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (!query_valid(w, queries[i])) return fail(w, DYN_ERR_INVALID, "dyn_query: a query record is invalid");
        queries[i].hit_base = (uint32_t)base;
        queries[i].count = 0u;
        queries[i].overflow = 0u;
        base += std::min(queries[i].max_hits, DYN_QUERY_CANDIDATES);
    }
    if (base > hit_capacity) return fail(w, DYN_ERR_CAPACITY, "dyn_query: the hit array is smaller than the batch's hit bound");
    if (w->states.empty()) return fail(w, DYN_ERR_INVALID, "dyn_query: the world holds no bodies");
    if (!w->dev || !w->dev->uploaded || (w->rows_dirty && !w->raw_rows) || w->scene_dirty) {
        if (dyn_status st = upload_scene(w)) return st;
    }
    DeviceState* d = w->dev;
    DYN_CUDA(cudaSetDevice(w->device));
    if (n > d->query_cap) {
        DYN_CUDA(cudaStreamSynchronize(d->stream));
        if (d->query_buf) cudaFree(d->query_buf);
        d->query_buf = nullptr;
        DYN_CUDA(cudaMalloc(&d->query_buf, (size_t)n * sizeof(dyn_query_record)));
        d->query_cap = n;
    }
    if (base > d->hit_cap) {
        DYN_CUDA(cudaStreamSynchronize(d->stream));
        if (d->hit_buf) cudaFree(d->hit_buf);
        d->hit_buf = nullptr;
        DYN_CUDA(cudaMalloc(&d->hit_buf, (size_t)std::max<uint64_t>(base, 1) * sizeof(dyn_query_hit_record)));
        d->hit_cap = (uint32_t)std::max<uint64_t>(base, 1);
    }
    // the grid of the current states, as a query run builds it (AABBs, entries, their sort, the cell table)
    dyn_step_params p;
    dyn_step_params_for(w, d->graph_dt > 0.0f ? d->graph_dt : 1.0f / 60.0f, &p);
    DeviceWorld dw = d->dw;
    const uint32_t K = std::max(dw.k, 1u), E = dw.e_cap;
    cudaStream_t s = d->stream;
    if (!d->query_entries) {
        DYN_CUDA(cudaStreamSynchronize(s));
        DYN_CUDA(cudaMalloc(&d->query_entries, 2 * (size_t)E * sizeof(float4)));
        DYN_CUDA(cudaMalloc(&d->query_words, (64 + CTL_COUNT) * sizeof(uint32_t)));
    }
    // the query's grid in its own entries, counters and control words (every collider in one run)
    dw.entries = d->query_entries;
    dw.counters = d->query_words;
    dw.ctl = d->query_words + 64;
    DYN_CUDA(cudaMemsetAsync(d->query_words, 0, (64 + CTL_COUNT) * sizeof(uint32_t), s));
    // the query's grid takes the merged list, cell table and run extents: the next step lists again
    DYN_CUDA(cudaMemsetAsync(d->dw.held + HELD_LIST_KEPT, 0, 2 * sizeof(uint32_t), s));
    k_aabb<<<blocks_for(d, K, 128), 128, 0, s>>>(dw, p);
    k_entry_count<false><<<blocks_for(d, K, 256), 256, 0, s>>>(dw);
    record_scan(d, s, dw.entry_count, dw.entry_offset, nullptr, dw.k, K, dw.ctl + CTL_ENTRIES);
    k_entry_emit<false><<<blocks_for(d, K, 256), 256, 0, s>>>(dw);
    record_sort(d, s, dw.ekey, nullptr, dw.eval, dw.ekey_alt, nullptr, dw.eval_alt, dw.ctl + CTL_ENTRIES, 0, E, 4, 0);
    k_cell_clear<<<blocks_for(d, 1u << dw.cell_bits, 256), 256, 0, s>>>(dw);
    k_cell_insert<<<blocks_for(d, E, 256), 256, 0, s>>>(dw);
    DYN_CUDA(cudaMemcpyAsync(d->query_buf, queries, (size_t)n * sizeof(dyn_query_record), cudaMemcpyHostToDevice, s));
    const size_t smem = sizeof(QueryShared);
    DYN_CUDA(cudaFuncSetAttribute(k_scene_query, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_scene_query<<<std::min<uint32_t>(n, d->sms * 4u), kQueryThreads, smem, s>>>(dw, d->query_buf, d->hit_buf, n);
    DYN_CUDA(cudaGetLastError());
    DYN_CUDA(cudaMemcpyAsync(queries, d->query_buf, (size_t)n * sizeof(dyn_query_record), cudaMemcpyDeviceToHost, s));
    if (base) DYN_CUDA(cudaMemcpyAsync(hits, d->hit_buf, (size_t)base * sizeof(dyn_query_hit_record), cudaMemcpyDeviceToHost, s));
    DYN_CUDA(cudaStreamSynchronize(s));
    return DYN_OK;
}

// The triangles of a hull source (index triples over its vertices, dyn_hull_info's order).
DYN_API dyn_status dyn_hull_triangles(const dyn_world* w, uint32_t source, uint32_t* out, uint32_t cap, uint32_t* count) {
    if (!w || source >= w->hulls.size()) return DYN_ERR_INVALID;
    const std::vector<uint32_t>& t = w->hulls[source].triangles;
    const uint32_t m = (uint32_t)(t.size() / 3);
    if (count) *count = m;
    if (out) std::memcpy(out, t.data(), (size_t)std::min(m, cap) * 3 * sizeof(uint32_t));
    return DYN_OK;
}

// The frozen contacts the next step reads (rest.cuh), six words each: first body id, its
// generation, second body id, its generation, collider a, collider b; in store order.
DYN_API dyn_status dyn_debug_resting(dyn_world* w, uint32_t* out, uint32_t cap, uint32_t* count) {
    if (!w || !w->dev) return DYN_ERR_INVALID;
    DeviceState* d = w->dev;
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    uint32_t live = 0;
    DYN_CUDA(cudaMemcpy(&live, d->dw.ctl + CTL_RESTING, 4, cudaMemcpyDeviceToHost));
    live = std::min(live, d->rest_cap);
    if (count) *count = live;
    if (!out || live == 0) return DYN_OK;
    const uint32_t m = std::min(live, cap);
    std::vector<uint4> ids(m);
    std::vector<uint2> slots(m);
    DYN_CUDA(cudaMemcpy(ids.data(), d->rest_ids[d->parity], m * sizeof(uint4), cudaMemcpyDeviceToHost));
    DYN_CUDA(cudaMemcpy(slots.data(), d->rest_slots[d->parity], m * sizeof(uint2), cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < m; ++i) {
        const uint32_t row[6] = {ids[i].x, ids[i].y, ids[i].z, ids[i].w, slots[i].x, slots[i].y};
        std::memcpy(out + 6 * (size_t)i, row, sizeof(row));
    }
    return DYN_OK;
}

DYN_API uint32_t dyn_step_kernel_count(const dyn_world* w) { return (w && w->dev) ? w->dev->graph_kernels : 0u; }

DYN_API dyn_status dyn_set_launch_config(dyn_world* w, const dyn_launch_config* c) {
    if (!w || !c) return DYN_ERR_INVALID;
    if (c->grid_blocks_per_sm < 1u || c->grid_blocks_per_sm > 64u || c->gjk_blocks_per_sm < 1u || c->gjk_blocks_per_sm > 16u ||
        c->epa_blocks_per_sm < 1u || c->epa_blocks_per_sm > 16u ||
        (c->solve_threads != 64u && c->solve_threads != 128u && c->solve_threads != 256u))
        return fail(w, DYN_ERR_INVALID, "dyn_set_launch_config: a field is out of its range");
    if (!w->dev) {
        w->launch = *c;
        return DYN_OK;
    }
    if (w->dev->tape.active) return fail(w, DYN_ERR_INVALID, "dyn_set_launch_config: a tape is recording");
    w->launch = *c;
    if (std::memcmp(&w->dev->launch, c, sizeof(*c)) != 0) {
        DYN_CUDA(cudaSetDevice(w->device));
        DYN_CUDA(cudaStreamSynchronize(w->dev->stream));
        w->dev->launch = *c;
        release_graphs(w->dev);  // the step graphs carry the launch shapes: record them again
    }
    return DYN_OK;
}
DYN_API dyn_status dyn_get_launch_config(const dyn_world* w, dyn_launch_config* out) {
    if (!w || !out) return DYN_ERR_INVALID;
    *out = w->dev ? w->dev->launch : w->launch;
    return DYN_OK;
}

// Coordinate descent over the launch shapes, each trial from the same checkpoint: every candidate
// value of one field with the others at their best so far, two rounds over the fields.
DYN_API dyn_status dyn_autotune(dyn_world* w, float dt, uint32_t steps, dyn_launch_config* best, float* best_ms) {
    if (!w || steps == 0u) return DYN_ERR_INVALID;
    if (!w->dev || !w->dev->uploaded) return fail(w, DYN_ERR_INVALID, "dyn_autotune: step the world once first");
    DeviceState* d = w->dev;
    if (d->tape.active) return fail(w, DYN_ERR_INVALID, "dyn_autotune: a tape is recording");
    if (!w->edits.empty()) return fail(w, DYN_ERR_INVALID, "dyn_autotune: body edits are queued");
    DYN_CUDA(cudaSetDevice(w->device));
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    Checkpoint saved;
    dyn_status st = save_checkpoint(w, &saved);
    if (st) return st;
    d->tuning = true;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    auto trial = [&](const dyn_launch_config& c, float* ms) -> dyn_status {
        dyn_status s2 = dyn_set_launch_config(w, &c);
        if (s2) return s2;
        if ((s2 = restore_checkpoint(w, saved))) return s2;
        if ((s2 = step_once(w, dt, false))) return s2;  // records the graph, warms the caches
        DYN_CUDA(cudaEventRecord(t0, d->stream));
        for (uint32_t k = 0; k < steps; ++k)
            if ((s2 = step_once(w, dt, false))) return s2;
        DYN_CUDA(cudaEventRecord(t1, d->stream));
        DYN_CUDA(cudaEventSynchronize(t1));
        DYN_CUDA(cudaEventElapsedTime(ms, t0, t1));
        *ms /= (float)steps;
        return DYN_OK;
    };
    dyn_launch_config top = d->launch;
    float top_ms = 0.0f;
    st = trial(top, &top_ms);
    const uint32_t grids[] = {4u, 8u, 16u, 32u}, threads[] = {64u, 128u, 256u}, gjks[] = {4u, 6u, 8u, 12u}, epas[] = {4u, 8u, 12u};
    for (int round = 0; round < 2 && !st; ++round) {
        for (int field = 0; field < 4 && !st; ++field) {
            const uint32_t* values = field == 0 ? grids : field == 1 ? threads : field == 2 ? gjks : epas;
            const int count = field == 1 || field == 3 ? 3 : 4;
            for (int v = 0; v < count && !st; ++v) {
                dyn_launch_config c = top;
                uint32_t* slot = field == 0 ? &c.grid_blocks_per_sm : field == 1 ? &c.solve_threads
                                 : field == 2 ? &c.gjk_blocks_per_sm : &c.epa_blocks_per_sm;
                if (*slot == values[v]) continue;
                *slot = values[v];
                float ms = 0.0f;
                st = trial(c, &ms);
                if (!st && ms < top_ms) {
                    top = c;
                    top_ms = ms;
                }
            }
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    d->tuning = false;
    if (!st) st = dyn_set_launch_config(w, &top);
    dyn_status restored = restore_checkpoint(w, saved);
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    free_checkpoint(&saved);
    if (st) return st;
    if (restored) return restored;
    if (best) *best = top;
    if (best_ms) *best_ms = top_ms;
    return DYN_OK;
}

// World::snapshot / World::restore (crates/dynamis-world/src/snapshot.rs:64-90): the simulated state
// of the world as it is once the queued steps finish (every body row and cold body field, the
// archived contacts the next step warm-starts from, the frozen contacts, the joints' runtime, the
// counters and control words, the contact-set parity), kept on the device, plus the body commands
// queued for the next step and the step clock. Restoring puts it back, so the steps that follow
// repeat the ones that followed the snapshot bit for bit. A snapshot belongs to the world it was
// taken from and to its scene: after a spawn, a removal, a constraint change or a contact-stream
// widening it is refused (DYN_ERR_INVALID); the reference carries its whole scene in the snapshot
// instead. Observations are abandoned on restore, as the reference's are.
struct dyn_snapshot {
    dyn_world* world = nullptr;
    dyn::DeviceState* dev = nullptr;
    uint64_t scene_epoch = 0;
    uint64_t steps_taken = 0;
    dyn::Checkpoint state;
    std::vector<uint32_t> edit_ids;
    std::vector<dyn_body_edit_record> edits;
};

DYN_API dyn_status dyn_snapshot_take(dyn_world* w, dyn_snapshot** out) {
    if (!w || !out) return DYN_ERR_INVALID;
    *out = nullptr;
    if (!w->dev || !w->dev->uploaded || (w->rows_dirty && !w->raw_rows) || w->scene_dirty || w->joints_dirty)
        return fail(w, DYN_ERR_INVALID, "dyn_snapshot_take: step the world (its current scene) once first");
    DeviceState* d = w->dev;
    if (d->tape.active) return fail(w, DYN_ERR_INVALID, "dyn_snapshot_take: a tape is recording");
    DYN_CUDA(cudaSetDevice(w->device));
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    dyn_snapshot* snap = new dyn_snapshot();
    if (dyn_status st = save_checkpoint(w, &snap->state)) {
        delete snap;
        return st;
    }
    if (cudaStreamSynchronize(d->stream) != cudaSuccess) {
        free_checkpoint(&snap->state);
        delete snap;
        return fail(w, DYN_ERR_CUDA, "dyn_snapshot_take: the copies failed");
    }
    snap->world = w;
    snap->dev = d;
    snap->scene_epoch = d->scene_epoch;
    snap->steps_taken = w->steps_taken;
    snap->edit_ids = w->edit_ids;
    snap->edits = w->edits;
    *out = snap;
    return DYN_OK;
}

DYN_API dyn_status dyn_snapshot_restore(dyn_world* w, const dyn_snapshot* snap) {
    if (!w || !snap) return DYN_ERR_INVALID;
    DeviceState* d = w->dev;
    if (snap->world != w || snap->dev != d || !d || d->scene_epoch != snap->scene_epoch || w->scene_dirty || w->joints_dirty ||
        (w->rows_dirty && !w->raw_rows))
        return fail(w, DYN_ERR_INVALID, "dyn_snapshot_restore: the snapshot belongs to another world or scene");
    if (d->tape.active) return fail(w, DYN_ERR_INVALID, "dyn_snapshot_restore: a tape is recording");
    if (checkpoint_bytes(checkpoint_parts(d)) != snap->state.bytes)
        return fail(w, DYN_ERR_INVALID, "dyn_snapshot_restore: the contact stream grew since the snapshot");
    DYN_CUDA(cudaSetDevice(w->device));
    if (dyn_status st = restore_checkpoint(w, snap->state)) return st;
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    for (uint32_t i = 0; i < kStepsInFlight; ++i) d->inflight_used[i] = false;
    w->edit_ids = snap->edit_ids;
    w->edits = snap->edits;
    w->steps_taken = snap->steps_taken;
    Observer& o = w->observer;
    for (ObservationSlot& slot : o.slots) {
        slot.pending = false;
        slot.ready = false;
    }
    o.latest = -1;
    return DYN_OK;
}

DYN_API dyn_status dyn_snapshot_free(dyn_snapshot* snap) {
    if (!snap) return DYN_OK;
    if (snap->state.base) {
        cudaFree(snap->state.base);
        snap->state.base = nullptr;
    }
    delete snap;
    return DYN_OK;
}

DYN_API dyn_status dyn_set_solver_guard(dyn_world* w, uint32_t flags) {
    if (!w) return DYN_ERR_INVALID;
    if (flags & ~DYN_SOLVER_GUARD_ROW_MASS) return fail(w, DYN_ERR_INVALID, "dyn_set_solver_guard: unknown flag");
    if (w->dev && w->dev->tape.active) return fail(w, DYN_ERR_INVALID, "dyn_set_solver_guard: a tape is recording");
    if (flags == w->solver_guard) return DYN_OK;
    w->solver_guard = flags;
    if (w->dev) {
        DYN_CUDA(cudaSetDevice(w->device));
        DYN_CUDA(cudaStreamSynchronize(w->dev->stream));
        release_graphs(w->dev);  // the step graphs carry the flag: record them again
    }
    return DYN_OK;
}

// World::set_ccd (crates/dynamis-world/src/body.rs:496-501): only a simulated body may declare
// continuous collision; a changed descriptor wakes the body (install_body, body.rs:284-290). The
// flag is patched into the device's body row in place, so the archived contacts and the simulated
// states stay; the step graph is recorded again when the world gains its first CCD body or loses
// its last.
DYN_API dyn_status dyn_set_ccd(dyn_world* w, uint32_t body_id, int32_t enabled) {
    if (!w) return DYN_ERR_INVALID;
    if (w->dev && w->dev->tape.active) return fail(w, DYN_ERR_INVALID, "dyn_set_ccd: a tape is recording");
    rebuild_rows(w);
    if (body_id >= w->row_of_id.size() || w->row_of_id[body_id] == DYN_NO_BODY)
        return fail(w, DYN_ERR_INVALID, "dyn_set_ccd: unknown body id");
    const uint32_t row = w->row_of_id[body_id];
    dyn_body_descriptor_record& desc = w->descs[row];
    if (enabled && !(desc.inverse_mass > 0.0f && (desc.flags & DYN_BODY_KINEMATIC) == 0u))
        return fail(w, DYN_ERR_INVALID, "dyn_set_ccd: only a simulated body can declare continuous collision");
    const uint32_t flags = enabled ? (desc.flags | DYN_BODY_CCD) : (desc.flags & ~DYN_BODY_CCD);
    if (flags == desc.flags) return DYN_OK;
    const bool gate_before = world_has_ccd(w);
    desc.flags = flags;
    if (body_id < w->spawn_descs.size()) w->spawn_descs[body_id].flags = flags;
    // rows or scene out of date: the next step uploads the scene, flags included
    if (w->dev && w->dev->uploaded && !w->scene_dirty && !(w->rows_dirty && !w->raw_rows)) {
        DeviceState* d = w->dev;
        DYN_CUDA(cudaSetDevice(w->device));
        DYN_CUDA(cudaStreamSynchronize(d->stream));
        DYN_CUDA(cudaMemcpy(&d->dw.hot[row].aux.y, &flags, sizeof(flags), cudaMemcpyHostToDevice));
        if (gate_before != world_has_ccd(w)) release_graphs(d);
    }
    dyn_body_edit_record wake{};
    wake.kind = DYN_EDIT_WAKE;
    w->edit_ids.push_back(body_id);
    w->edits.push_back(wake);
    return DYN_OK;
}

DYN_API dyn_status dyn_set_timing(dyn_world* w, int32_t enabled) {
    if (!w) return DYN_ERR_INVALID;
    w->timing = enabled != 0;
    return DYN_OK;
}
DYN_API uint32_t dyn_stage_count(void) { return ST_COUNT; }
DYN_API const char* dyn_stage_name(uint32_t stage) { return stage < ST_COUNT ? kStageNames[stage] : ""; }
DYN_API dyn_status dyn_stage_timings(dyn_world* w, float* ms, uint32_t n) {
    if (!w || !ms || !w->dev) return DYN_ERR_INVALID;
    DeviceState* d = w->dev;
    DYN_CUDA(cudaStreamSynchronize(d->stream));
    float acc[ST_COUNT] = {0};
    for (size_t i = 0; i + 1 < d->events.size(); ++i) {
        float t = 0.0f;
        DYN_CUDA(cudaEventElapsedTime(&t, d->events[i], d->events[i + 1]));
        uint32_t stage = d->event_stage[i];
        if (stage < ST_COUNT) acc[stage] += t;
    }
    for (uint32_t i = 0; i < std::min<uint32_t>(n, ST_COUNT); ++i) ms[i] = acc[i];
    return DYN_OK;
}

DYN_API dyn_status dyn_radix_sort(dyn_world* w, uint32_t* major, uint32_t* minor, uint32_t* payload, uint32_t n,
                                  uint32_t major_digits, uint32_t minor_digits) {
    if (!w || !major || major_digits > 4 || minor_digits > 4 || (minor_digits && !minor)) return DYN_ERR_INVALID;
    if (n == 0 || major_digits + minor_digits == 0) return DYN_OK;
    if (!w->dev) {
        dyn_status st = ensure_device(w);
        if (st) return st;
    }
    DeviceState* d = w->dev;
    if (d->sort_alt_cap < n) {
        for (uint32_t** p : {&d->sort_alt0, &d->sort_alt1, &d->sort_alt2}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
        d->sort_alt_cap = 0;
        // owned here (freed on growth and in destroy_device), not in the world's allocation list
        DYN_CUDA(cudaMalloc(&d->sort_alt0, (size_t)n * 4));
        DYN_CUDA(cudaMalloc(&d->sort_alt1, (size_t)n * 4));
        DYN_CUDA(cudaMalloc(&d->sort_alt2, (size_t)n * 4));
        d->sort_alt_cap = n;
    }
    uint32_t tiles = div_up(n, kSortTile);
    if ((size_t)(major_digits + minor_digits) * tiles * 256 > d->lookback_words) {
        return fail(w, DYN_ERR_CAPACITY, "dyn_radix_sort: more keys than the world's sort scratch holds");
    }
    const uint32_t limit = d->sort_fault_armed ? d->sort_fault_limit : kLookbackSpinLimit;
    const uint32_t first_ticket = d->sort_fault_armed ? d->sort_fault_skip : 0u;
    d->sort_fault_armed = false;
    record_sort(d, d->stream, major, minor, payload, d->sort_alt0, minor ? d->sort_alt1 : nullptr,
                payload ? d->sort_alt2 : nullptr, nullptr, n, n, major_digits, minor_digits, limit, first_ticket);
    DYN_CUDA(cudaGetLastError());
    return DYN_OK;
}

DYN_API dyn_status dyn_debug_sort_fault(dyn_world* w, uint32_t skipped_tiles, uint32_t spin_limit) {
    if (!w) return static_sort_fault(skipped_tiles, spin_limit);
    if (spin_limit == 0u || skipped_tiles > 1u) return fail(w, DYN_ERR_INVALID, "dyn_debug_sort_fault: spin_limit must be > 0, skipped_tiles 0 or 1");
    if (!w->dev) {
        dyn_status st = ensure_device(w);
        if (st) return st;
    }
    w->dev->sort_fault_armed = true;
    w->dev->sort_fault_skip = skipped_tiles;
    w->dev->sort_fault_limit = spin_limit;
    return DYN_OK;
}

DYN_API dyn_status dyn_clear_device_status(dyn_world* w) {
    if (!w) return DYN_ERR_INVALID;
    if (!w->dev) return DYN_OK;
    DYN_CUDA(cudaStreamSynchronize(w->dev->stream));
    DYN_CUDA(cudaMemsetAsync(w->dev->dw.ctl + CTL_STATUS, 0, 4, w->dev->stream));
    DYN_CUDA(cudaStreamSynchronize(w->dev->stream));
    return DYN_OK;
}

}  // extern "C"
