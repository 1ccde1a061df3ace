"""World: the host-side mirror of dynamis-world's World over the C ABI.

Method names follow crates/dynamis-world/src (World::new lib.rs:86, spawn body.rs:108,
add_hull_from_mesh shape.rs:50, step step.rs:34, wait observation.rs:484, read_state body.rs:326,
measured readback.rs:215, refusals readback.rs:226). Invalid input raises (the reference panics).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import records as R
from ._native import DynamisError, check, lib, ptr

NOT_READY = 7  # DYN_NOT_READY: no observation has completed yet


def default_config() -> np.ndarray:
    c = np.zeros(1, R.CONFIG)
    lib.dyn_config_default(ptr(c))
    return c


class World:
    """One simulated world on one GPU (crates/dynamis-world/src/lib.rs:64-109)."""

    def __init__(self, config: np.ndarray | None = None, capacity: dict | None = None, device: int = 0, **overrides):
        cfg = default_config() if config is None else np.array(config, R.CONFIG).reshape(1)
        for key, value in overrides.items():
            cfg[key] = value
        cap = np.zeros(1, R.CAPACITY)
        for key, value in (capacity or {}).items():
            cap[key] = value
        handle = ctypes.c_void_p()
        check(lib.dyn_world_create(ptr(cfg), ptr(cap), int(device), ctypes.byref(handle)))
        self._h = handle
        self.config = cfg

    def close(self) -> None:
        if self._h:
            lib.dyn_world_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status: int) -> None:
        check(status, self._h)

    # ---- scene ----
    def add_hull(self, points) -> int:
        """The convex hull of a point cloud (add_hull_from_mesh with every point referenced)."""
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = ctypes.c_uint32()
        self._check(lib.dyn_add_hull(self._h, ptr(pts), len(pts), ctypes.byref(out)))
        return out.value

    def add_hull_from_mesh(self, vertices, triangles) -> int:
        """World::add_hull_from_mesh: the convex hull of the vertices the triangles reference."""
        pts = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        tris = np.ascontiguousarray(triangles, np.uint32).reshape(-1, 3)
        out = ctypes.c_uint32()
        self._check(lib.dyn_add_hull_from_mesh(self._h, ptr(pts), len(pts), ptr(tris), len(tris), ctypes.byref(out)))
        return out.value

    def add_hull_mesh(self, vertices, triangles) -> int:
        """World::add_hull: a hull given as its own vertices and outward triangles."""
        pts = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        tris = np.ascontiguousarray(triangles, np.uint32).reshape(-1, 3)
        out = ctypes.c_uint32()
        self._check(lib.dyn_add_hull_mesh(self._h, ptr(pts), len(pts), ptr(tris), len(tris), ctypes.byref(out)))
        return out.value

    def hull_info(self, source: int) -> dict:
        vc, tc, vol = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_float()
        cen = np.zeros(3, np.float32)
        self._check(lib.dyn_hull_info(self._h, source, ctypes.byref(vc), ctypes.byref(tc), ctypes.byref(vol), ptr(cen)))
        return {"vertices": vc.value, "triangles": tc.value, "volume": vol.value, "centroid": cen}

    def spawn(self, bodies: np.ndarray, colliders: np.ndarray) -> np.ndarray:
        """World::spawn for every BODY_DESC row; returns the body ids."""
        bodies = np.ascontiguousarray(bodies, R.BODY_DESC)
        colliders = np.ascontiguousarray(colliders, R.COLLIDER_DESC)
        ids = np.zeros(len(bodies), np.uint32)
        self._check(lib.dyn_spawn_bodies(self._h, ptr(bodies), len(bodies), ptr(colliders), len(colliders), ptr(ids)))
        return ids

    def upload_bodies(self, states, descs, colliders, owners) -> None:
        states = np.ascontiguousarray(states, R.BODY_STATE)
        descs = np.ascontiguousarray(descs, R.BODY_DESCRIPTOR)
        colliders = np.ascontiguousarray(colliders, R.COLLIDER)
        owners = np.ascontiguousarray(owners, np.uint32)
        self._check(lib.dyn_upload_bodies(self._h, ptr(states), ptr(descs), len(states), ptr(colliders), ptr(owners),
                                          len(colliders)))

    def upload_states(self, states: np.ndarray) -> None:
        states = np.ascontiguousarray(states, R.BODY_STATE)
        self._check(lib.dyn_upload_states(self._h, ptr(states), len(states)))

    def stream_capacity(self) -> dict:
        """The device's pair and contact stream capacities (World::stream_capacity); 0 before the first
        step. The pair stream widens by itself after a step that refused pairs."""
        pairs, contacts = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(lib.dyn_stream_capacity(self._h, ctypes.byref(pairs), ctypes.byref(contacts)))
        return {"pairs": pairs.value, "contacts": contacts.value}

    def sizes(self) -> dict:
        vals = [ctypes.c_uint32() for _ in range(5)]
        self._check(lib.dyn_scene_sizes(self._h, *[ctypes.byref(v) for v in vals]))
        return dict(zip(["bodies", "dynamic", "colliders", "sources", "vertices"], [v.value for v in vals]))

    def export_scene(self) -> dict:
        """The scene as rows: the exact records the device receives."""
        s = self.sizes()
        states = np.zeros(s["bodies"], R.BODY_STATE)
        descs = np.zeros(s["bodies"], R.BODY_DESCRIPTOR)
        colliders = np.zeros(s["colliders"], R.COLLIDER)
        owners = np.zeros(s["colliders"], np.uint32)
        sources = np.zeros(s["sources"], R.SHAPE_SOURCE)
        vertices = np.zeros((max(s["vertices"], 0), 4), np.float32)
        self._check(lib.dyn_export_scene(self._h, ptr(states), ptr(descs), ptr(colliders), ptr(owners), ptr(sources),
                                         ptr(vertices)))
        scene = {"states": states, "descs": descs, "colliders": colliders, "owners": owners, "sources": sources,
                 "vertices": vertices, "dynamic": s["dynamic"],
                 "hull_triangles": [self.hull_triangles(i) for i in range(s["sources"])]}
        body_world = np.zeros(s["bodies"], np.uint32)
        self._check(lib.dyn_export_body_worlds(self._h, ptr(body_world)))
        if body_world.any():
            scene["body_world"] = body_world
        m = self.constraint_count()
        if m:
            jd, jr, jt = np.zeros(m, R.CONSTRAINT_DESCRIPTOR), np.zeros(m, R.CONSTRAINT_ROWS), np.zeros(m, R.CONSTRAINT_RUNTIME)
            self._check(lib.dyn_export_constraints(self._h, ptr(jd), ptr(jr), ptr(jt)))
            scene.update(constraint_descs=jd, constraint_rows=jr, constraint_runtime=jt)
        return scene

    # ---- batched worlds ----
    def set_body_worlds(self, world_of_body) -> None:
        """Puts every body (indexed by body id) in a sub-world; sub-worlds never interact."""
        arr = np.ascontiguousarray(world_of_body, np.uint32)
        self._check(lib.dyn_set_body_worlds(self._h, ptr(arr), len(arr)))

    # ---- lagged observations ----
    def observe_bodies(self, body_ids=None) -> None:
        """World::observe_bodies (or observe_all_bodies when body_ids is None)."""
        if body_ids is None:
            self._check(lib.dyn_observe_bodies(self._h, None, 0))
        else:
            ids = np.ascontiguousarray(body_ids, np.uint32)
            self._check(lib.dyn_observe_bodies(self._h, ptr(ids), len(ids)))

    def stop_observing(self) -> None:
        self._check(lib.dyn_stop_observing(self._h))

    def poll(self) -> None:
        self._check(lib.dyn_poll(self._h))

    def try_state(self, body_id: int):
        """World::try_state: (state record, step it was taken after) from the newest completed
        observation, or None while none has completed. Never waits for the GPU."""
        out = np.zeros(1, R.BODY_STATE)
        step = ctypes.c_uint64()
        status = lib.dyn_try_state(self._h, int(body_id), ptr(out), ctypes.byref(step))
        if status == NOT_READY:
            return None
        self._check(status)
        return out[0], step.value

    def try_counters(self):
        out = np.zeros(R.COUNTER_DEVICE_COUNT, np.uint32)
        step = ctypes.c_uint64()
        status = lib.dyn_try_counters(self._h, ptr(out), len(out), ctypes.byref(step))
        if status == NOT_READY:
            return None
        self._check(status)
        return out, step.value

    def remove_bodies(self, body_ids) -> None:
        """World::remove for each id: the bodies leave the world at the next step."""
        ids = np.ascontiguousarray(body_ids, np.uint32)
        self._check(lib.dyn_remove_bodies(self._h, ptr(ids), len(ids)))

    # ---- body commands ----
    def edit_bodies(self, body_ids, edits: np.ndarray) -> None:
        """Queues BodyEdit records (records.BODY_EDIT) for the next step, one per body id; a body's
        commands run in the order given, after the step clears the applied forces."""
        ids = np.ascontiguousarray(body_ids, np.uint32)
        recs = np.ascontiguousarray(edits, R.BODY_EDIT)
        if len(ids) != len(recs):
            raise ValueError("one body id per edit")
        self._check(lib.dyn_edit_bodies(self._h, ptr(ids), ptr(recs), len(ids)))

    def apply_force(self, body_id: int, force) -> None:
        self.edit_bodies([body_id], R.body_edit(R.EDIT_FORCE, force=force))

    def apply_impulse(self, body_id: int, impulse, point=None) -> None:
        if point is None:
            self.edit_bodies([body_id], R.body_edit(R.EDIT_IMPULSE, velocity=impulse))
        else:
            self.edit_bodies([body_id], R.body_edit(R.EDIT_IMPULSE_AT_POINT, velocity=impulse, position=point))

    def teleport(self, body_id: int, position=None, orientation=None) -> None:
        mask = (R.PATCH_POSITION if position is not None else 0) | (R.PATCH_ORIENTATION if orientation is not None else 0)
        self.edit_bodies([body_id], R.body_edit(R.EDIT_PATCH, mask=mask, position=position, orientation=orientation))

    def sleep_body(self, body_id: int) -> None:
        self.edit_bodies([body_id], R.body_edit(R.EDIT_SLEEP))

    def wake_body(self, body_id: int) -> None:
        self.edit_bodies([body_id], R.body_edit(R.EDIT_WAKE))

    # ---- constraints ----
    def add_ball_joint(self, first_body: int, second_body: int, anchor_a, anchor_b) -> int:
        """World::add_constraint(first, second, ConstraintDesc::ball(anchor_a, anchor_b)); returns the id."""
        a = np.ascontiguousarray(anchor_a, np.float32)
        b = np.ascontiguousarray(anchor_b, np.float32)
        out = ctypes.c_uint32()
        self._check(lib.dyn_add_ball_joint(self._h, int(first_body), int(second_body), ptr(a), ptr(b), ctypes.byref(out)))
        return out.value

    def add_constraints(self, records: np.ndarray) -> int:
        """Appends ConstraintDescriptorRecords; returns the id of the first."""
        records = np.ascontiguousarray(records, R.CONSTRAINT_DESCRIPTOR)
        out = ctypes.c_uint32()
        self._check(lib.dyn_add_constraints(self._h, ptr(records), len(records), ctypes.byref(out)))
        return out.value

    def constraint_count(self) -> int:
        out = ctypes.c_uint32()
        self._check(lib.dyn_constraint_count(self._h, ctypes.byref(out)))
        return out.value

    def read_constraints(self) -> np.ndarray:
        """ConstraintRuntimeRecords after the last step (accumulated impulses, reactions, broken)."""
        m = self.constraint_count()
        out = np.zeros(m, R.CONSTRAINT_RUNTIME)
        self._check(lib.dyn_read_constraints(self._h, ptr(out), m))
        return out

    def joint_plan(self) -> dict:
        """The joint solve order: rows, (first, count) layers and (first layer, count) components."""
        nl, nc = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(lib.dyn_joint_plan(self._h, None, None, None, ctypes.byref(nl), ctypes.byref(nc)))
        rows = np.zeros(self.constraint_count(), np.uint32)
        layers = np.zeros((nl.value, 2), np.uint32)
        comps = np.zeros((nc.value, 2), np.uint32)
        self._check(lib.dyn_joint_plan(self._h, ptr(rows), ptr(layers), ptr(comps), None, None))
        return {"rows": rows, "layers": layers, "components": comps}

    def launch_config(self) -> dict:
        """dyn_get_launch_config: the launch shapes the step uses."""
        c = np.zeros(1, R.LAUNCH_CONFIG)
        self._check(lib.dyn_get_launch_config(self._h, ptr(c)))
        return {k: int(c[k][0]) for k in R.LAUNCH_CONFIG.names}

    def set_launch_config(self, **fields) -> None:
        """dyn_set_launch_config: change any of the launch shapes (no result changes)."""
        c = np.zeros(1, R.LAUNCH_CONFIG)
        for k, v in {**self.launch_config(), **fields}.items():
            c[k] = v
        self._check(lib.dyn_set_launch_config(self._h, ptr(c)))

    def autotune(self, dt: float, steps: int = 3) -> tuple[dict, float]:
        """dyn_autotune: the fastest launch shapes for this world as it stands (kept), with their
        device time per step in ms; the world's state is left as it was."""
        c = np.zeros(1, R.LAUNCH_CONFIG)
        ms = ctypes.c_float()
        self._check(lib.dyn_autotune(self._h, float(dt), int(steps), ptr(c), ctypes.byref(ms)))
        return {k: int(c[k][0]) for k in R.LAUNCH_CONFIG.names}, ms.value

    def snapshot(self) -> "Snapshot":
        """World::snapshot: the simulated state once the queued steps finish (dyn_snapshot_take)."""
        handle = ctypes.c_void_p()
        self._check(lib.dyn_snapshot_take(self._h, ctypes.byref(handle)))
        return Snapshot(handle)

    def restore(self, snapshot: "Snapshot") -> None:
        """World::restore: back to the snapshot's state; later steps repeat the ones that followed it."""
        self._check(lib.dyn_snapshot_restore(self._h, snapshot._h))

    def set_solver_guard(self, flags: int) -> None:
        """dyn_set_solver_guard: SOLVER_GUARD_ROW_MASS keeps every contact block's Jacobi iteration
        convergent where the reference's manifold row masses would let it diverge; 0 (the default)
        is the reference's solver."""
        self._check(lib.dyn_set_solver_guard(self._h, int(flags)))

    def set_ccd(self, body_id: int, enabled: bool = True) -> None:
        """dyn_set_ccd (World::set_ccd): declares or clears continuous collision for a simulated body;
        a changed flag wakes the body at the next step."""
        self._check(lib.dyn_set_ccd(self._h, int(body_id), 1 if enabled else 0))

    def step_params(self, dt: float) -> np.ndarray:
        p = np.zeros(1, R.STEP_PARAMS)
        self._check(lib.dyn_step_params_for(self._h, float(dt), ptr(p)))
        return p

    # ---- stepping ----
    def step(self, dt: float) -> None:
        """World::step: enqueues one step; returns without waiting."""
        self._check(lib.dyn_step(self._h, float(dt)))

    def wait(self) -> None:
        """World::wait: blocks until queued steps finish; raises on a sticky device status."""
        self._check(lib.dyn_sync(self._h))

    def set_stream(self, cuda_stream: int | None) -> None:
        self._check(lib.dyn_world_set_stream(self._h, cuda_stream))

    # ---- readback ----
    def read_states(self) -> np.ndarray:
        """All body states in row order (dynamic rows first)."""
        n = self.sizes()["bodies"]
        out = np.zeros(n, R.BODY_STATE)
        self._check(lib.dyn_download_states(self._h, ptr(out), n))
        return out

    def read_state(self, body_id: int) -> np.ndarray:
        out = np.zeros(1, R.BODY_STATE)
        self._check(lib.dyn_read_state(self._h, int(body_id), ptr(out)))
        return out[0]

    def measured(self) -> np.ndarray:
        out = np.zeros(R.COUNTER_DEVICE_COUNT, np.uint32)
        self._check(lib.dyn_read_counters(self._h, ptr(out), len(out)))
        return out

    def refusals(self) -> dict:
        m = self.measured()
        names = ["REFUSED_PAIRS", "REFUSED_CONTACTS", "ENTRY_FAULTS", "ISLAND_FAULTS", "LIVE_FAULTS"]
        return {n: int(m[R.COUNTER[n]]) for n in names}

    # ---- parity hooks (the last step's intermediate products) ----
    def debug_aabbs(self) -> np.ndarray:
        n = ctypes.c_uint32()
        self._check(lib.dyn_debug_aabbs(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, R.AABB)
        self._check(lib.dyn_debug_aabbs(self._h, ptr(out), n.value, None))
        return out

    def debug_entries(self):
        n = ctypes.c_uint32()
        self._check(lib.dyn_debug_entries(self._h, None, None, 0, ctypes.byref(n)))
        keys = np.zeros(n.value, np.uint32)
        infos = np.zeros(n.value, np.uint32)
        self._check(lib.dyn_debug_entries(self._h, ptr(keys), ptr(infos), n.value, None))
        return keys, infos

    def debug_pairs(self):
        n = ctypes.c_uint32()
        self._check(lib.dyn_debug_pairs(self._h, None, None, 0, ctypes.byref(n)))
        major = np.zeros(n.value, np.uint32)
        minor = np.zeros(n.value, np.uint32)
        self._check(lib.dyn_debug_pairs(self._h, ptr(major), ptr(minor), n.value, None))
        return major, minor

    def debug_contacts(self) -> np.ndarray:
        n = ctypes.c_uint32()
        self._check(lib.dyn_debug_contacts(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, R.CONTACT)
        self._check(lib.dyn_debug_contacts(self._h, ptr(out), n.value, None))
        return out

    def debug_islands(self) -> np.ndarray:
        n = ctypes.c_uint32()
        self._check(lib.dyn_debug_islands(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, np.uint32)
        self._check(lib.dyn_debug_islands(self._h, ptr(out), n.value, None))
        return out

    def query(self, queries: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """dyn_query: a batch of scene queries (records.QUERY, e.g. from records.ray_query) against the
        current states. Returns the records (hit_base, count and overflow set) and the hit array
        (records.QUERY_HIT); query i's hits are hits[hit_base : hit_base + count], nearest first."""
        q = np.array(queries, R.QUERY).reshape(-1)
        bound = int(np.minimum(q["max_hits"], R.QUERY_CANDIDATES).sum())
        hits = np.zeros(max(bound, 1), R.QUERY_HIT)
        self._check(lib.dyn_query(self._h, ptr(q), len(q), ptr(hits), len(hits)))
        return q, hits[:bound]

    def hull_triangles(self, source: int) -> np.ndarray:
        """dyn_hull_triangles: the hull's triangles, (m, 3) vertex indices."""
        n = ctypes.c_uint32()
        self._check(lib.dyn_hull_triangles(self._h, int(source), None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 3), np.uint32)
        if n.value:
            self._check(lib.dyn_hull_triangles(self._h, int(source), ptr(out), n.value, None))
        return out

    def debug_resting(self) -> np.ndarray:
        """The frozen contacts the next step reads, one row each: first body id, its generation,
        second body id, its generation, collider a, collider b (store order)."""
        n = ctypes.c_uint32()
        self._check(lib.dyn_debug_resting(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 6), np.uint32)
        if n.value:
            self._check(lib.dyn_debug_resting(self._h, ptr(out), n.value, None))
        return out

    # ---- differentiation (World::step_backward) ----
    def set_mass_properties(self, inverse_mass, inverse_inertia) -> None:
        """Every body row's inverse mass and inverse inertia tensor (rows x 6: xx, xy, xz, yy, yz, zz)."""
        im = np.ascontiguousarray(inverse_mass, np.float32)
        ii = np.ascontiguousarray(inverse_inertia, np.float32).reshape(len(im), 6)
        self._check(lib.dyn_set_mass_properties(self._h, ptr(im), ptr(ii), len(im)))

    def set_friction(self, friction) -> None:
        """Every collider's friction, in dyn_export_scene's collider order."""
        f = np.ascontiguousarray(friction, np.float32)
        self._check(lib.dyn_set_friction(self._h, ptr(f), len(f)))

    def tape_begin(self, checkpoint_interval: int = 10) -> None:
        """Starts recording a differentiable trajectory (checkpoints every `checkpoint_interval` steps)."""
        self._check(lib.dyn_tape_begin(self._h, int(checkpoint_interval)))

    def tape_end(self) -> None:
        """Restores the state after the last recorded step and releases the tape."""
        self._check(lib.dyn_tape_end(self._h))

    def tape_steps(self) -> tuple:
        rec, rev = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(lib.dyn_tape_steps(self._h, ctypes.byref(rec), ctypes.byref(rev)))
        return rec.value, rev.value

    def step_backward(self, grad: np.ndarray, steps: int = 1) -> np.ndarray:
        """World::step_backward over `steps` recorded steps: `grad` (BODY_GRAD per row) is d loss / d
        state after the last unreversed step; returns d loss / d state its earliest reversed step's
        solve started from."""
        g = np.ascontiguousarray(grad, R.BODY_GRAD)
        out = np.zeros(len(g), R.BODY_GRAD)
        self._check(lib.dyn_backward(self._h, ptr(g), ptr(out), len(g), int(steps)))
        return out

    def param_grads(self) -> dict:
        """Accumulated d loss / d inverse mass and d loss / d inverse-inertia scale per row, d loss / d
        friction per collider."""
        sizes = self.sizes()
        n, k = sizes["bodies"], sizes["colliders"]
        im, sc, fr = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(k, np.float32)
        self._check(lib.dyn_param_grads(self._h, ptr(im), ptr(sc), n, ptr(fr), k))
        return {"inverse_mass": im, "inertia_scale": sc, "friction": fr}

    # ---- timing ----
    def step_kernel_count(self) -> int:
        """Kernel launches per step (kernel nodes of the captured step graph)."""
        return int(lib.dyn_step_kernel_count(self._h))

    def set_timing(self, enabled: bool) -> None:
        self._check(lib.dyn_set_timing(self._h, 1 if enabled else 0))

    def stage_timings(self) -> dict:
        n = lib.dyn_stage_count()
        ms = np.zeros(n, np.float32)
        self._check(lib.dyn_stage_timings(self._h, ptr(ms), n))
        return {lib.dyn_stage_name(i).decode(): float(ms[i]) for i in range(n)}


__all__ = ["World", "DynamisError", "default_config"]


class Snapshot:
    """A world's device-side snapshot (dyn_snapshot); freed when closed or collected."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle

    def close(self) -> None:
        if self._h:
            lib.dyn_snapshot_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
