// rest.cuh - frozen contacts: the contacts of body pairs that were both at rest when a step ended
// stay in a store across steps, keep the sleeping bodies they join in one island, and are released
// once either body moves again (crates/dynamis-rigid/shaders/freeze_contacts.wgsl,
// thaw_contacts.wgsl, island_link_resting.wgsl; the commit order of crates/dynamis-rigid/src/
// commit.rs:187-208: thaw, archive, static_wake_clear, freeze).
//
// The reference keeps its resting contacts in slots taken from a free list (atomic compare-exchange)
// and flags them live; here the store is rewritten every step, so it is always compact: the commit
// appends the contacts that stay frozen, then the newly frozen ones, into the other of two stores.
// Their order is the order the appends land in, which changes nothing the store feeds: island
// unions by minimum row and the wake carried from a static row do not depend on it. COUNTER_RESTING
// is the reference's slot count: with a free list, slots are added only when the live contacts
// outnumber them, so it is the largest number of contacts held frozen at once.
#pragma once

#include "step.cuh"

namespace dyn {

__device__ __forceinline__ bool row_active(const DeviceWorld& w, uint32_t row) {
    const BodyHot& h = w.hot[row];
    return moves(h.pos.w, h.aux.y) && h.aux.x == 0u;  // body_is_active, core.wgsl:229-231
}

// island_link_resting.wgsl runs inside the second contact-link pass (k_island_link<false>, step.cuh).

// thaw_contacts.wgsl:47-76: a frozen contact stays while both of its bodies were inactive when the
// step began (activity.wgsl, written by k_begin); one whose body is gone is released and its other
// body disturbed (a wake flag the next step acts on). Contact events are not published here.
// The same launch clears the static rows' wake flags (static_wake_clear.wgsl), which the reference
// runs right after the thaw: a disturbed static row would lose its flag there at once, so the thaw
// here disturbs dynamic rows only, and the two loops need no order between them.
__global__ void k_rest_thaw(DeviceWorld w) {
    const uint32_t statics = w.n - w.nd;
    GRID_STRIDE(i, statics) w.wake_flags[w.nd + i] = 0u;
    const uint32_t count = min(w.ctl[CTL_RESTING], w.rest_cap);
    GRID_STRIDE(i, count) {
        const uint4 r = w.rest_in[i];
        const uint32_t a = resolve_row(w, r.x, r.y), b = resolve_row(w, r.z, r.w);
        if (a == DYN_NO_BODY || b == DYN_NO_BODY) {
            if (a != DYN_NO_BODY && a < w.nd) atomicOr(&w.wake_flags[a], 1u);
            if (b != DYN_NO_BODY && b < w.nd) atomicOr(&w.wake_flags[b], 1u);
            continue;
        }
        if (w.activity[a] != 0u || w.activity[b] != 0u) continue;
        const uint32_t slot = append_slot(&w.ctl[CTL_REST_NEXT]);
        if (slot >= w.rest_cap) continue;  // the kept ones never outnumber the store they came from
        w.rest_out[slot] = r;
        w.rest_out_slots[slot] = w.rest_in_slots[i];
    }
}

// freeze_contacts.wgsl:29-45: every contact of this step whose bodies are both inactive after it
// (asleep or static) is frozen; past the store's capacity it is refused and counted.
__global__ void k_rest_freeze(DeviceWorld w) {
    const uint32_t count = w.ctl[CTL_CONTACTS];
    GRID_STRIDE(i, count) {
        const uint4 r = w.cur.rows[i];
        if (row_active(w, r.x) || row_active(w, r.y)) continue;
        const uint4 ids = w.cur.ids[i], ids2 = w.cur.ids2[i];
        const uint32_t slot = append_slot(&w.ctl[CTL_REST_NEXT]);
        if (slot >= w.rest_cap) {
            add_counter(&w.counters[DYN_COUNTER_REFUSED_RESTING], 1u);
            continue;
        }
        w.rest_out[slot] = make_uint4(ids.z, ids2.x, ids.w, ids2.y);
        w.rest_out_slots[slot] = make_uint2(ids.x, ids.y);
    }
}

// The store the next step reads, and COUNTER_RESTING (the most contacts held frozen at once).
__global__ void k_rest_commit(DeviceWorld w) {
    const uint32_t live = min(w.ctl[CTL_REST_NEXT], w.rest_cap);
    w.ctl[CTL_RESTING] = live;
    if (live > w.counters[DYN_COUNTER_RESTING]) w.counters[DYN_COUNTER_RESTING] = live;
}

}  // namespace dyn
