"""ctypes wrapper of the oracle library (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker used by tests/ and bench.py's cpu_baseline leg. It runs the
CPU restatement of the Dynamis step (oracle.cpp) on records exported from a dynamis_b200 World, or
on records it builds itself from the scene's descriptions (scene.cpp: the reference's spawn path).
"""
from __future__ import annotations

import ctypes

import numpy as np

from dynamis_b200 import records as R

from .build import build

_lib = None
P = ctypes.c_void_p
U32 = ctypes.c_uint32


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(build()))
        _lib.orc_world_create.restype = P
        _lib.orc_world_create.argtypes = [P, P, P, U32, P, P, U32, P, U32, P, U32, U32, U32]
        _lib.orc_world_destroy.argtypes = [P]
        _lib.orc_step.argtypes = [P, ctypes.c_float]
        _lib.orc_counters.argtypes = [P, P]
        for name in ("orc_states", "orc_aabbs", "orc_contacts", "orc_islands"):
            getattr(_lib, name).restype = U32
            getattr(_lib, name).argtypes = [P, P]
        _lib.orc_entry_keys.restype = U32
        _lib.orc_entry_keys.argtypes = [P, P, P]
        _lib.orc_pairs.restype = U32
        _lib.orc_pairs.argtypes = [P, P, P]
        for name in ("orc_sin", "orc_cos"):
            getattr(_lib, name).restype = ctypes.c_float
            getattr(_lib, name).argtypes = [ctypes.c_float]
        _lib.orc_atan2.restype = ctypes.c_float
        _lib.orc_atan2.argtypes = [ctypes.c_float, ctypes.c_float]
        _lib.orc_key_words.restype = U32
        _lib.orc_key_words.argtypes = [U32]
        _lib.orc_radix_sort.argtypes = [P, P, P, U32, U32, U32]
        _lib.orc_narrowphase_pair.restype = U32
        _lib.orc_narrowphase_pair.argtypes = [P, U32, U32, P]
        _lib.orc_set_constraints.restype = U32
        _lib.orc_set_constraints.argtypes = [P, P, P, P, U32]
        _lib.orc_constraints.restype = U32
        _lib.orc_constraints.argtypes = [P, P]
        _lib.orc_joint_plan.argtypes = [P, P, P, P, P]
        _lib.orc_set_body_worlds.argtypes = [P, P, U32]
        _lib.orc_queue_edits.argtypes = [P, P, P, U32]
        _lib.orc_threads.restype = U32
        _lib.orc_set_threads.argtypes = [U32]
        _lib.orc_config_default.argtypes = [P]
        _lib.orc_hull_from_mesh.restype = U32
        _lib.orc_hull_from_mesh.argtypes = [P, U32, P, U32, P, P, U32, P]
        _lib.orc_scene_build.restype = P
        _lib.orc_scene_build.argtypes = [P, P, P, P, P, U32, P, U32, P, U32]
        _lib.orc_scene_error.restype = ctypes.c_int
        _lib.orc_scene_error.argtypes = [P]
        _lib.orc_scene_free.argtypes = [P]
        _lib.orc_scene_sizes.argtypes = [P, P, P, P, P, P]
        _lib.orc_scene_export.argtypes = [P, P, P, P, P, P, P]
        _lib.orc_scene_params.argtypes = [P, ctypes.c_float, P]
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


class OracleWorld:
    """The CPU restatement of one world, built from exported scene records."""

    def __init__(self, scene: dict, params: np.ndarray, pair_capacity: int = 1 << 26, contact_capacity: int = 1 << 25):
        L = lib()
        self._keep = {k: np.ascontiguousarray(v) for k, v in scene.items() if isinstance(v, np.ndarray)}
        s = self._keep
        self.n = len(s["states"])
        self._h = L.orc_world_create(_p(np.ascontiguousarray(params, R.STEP_PARAMS)), _p(s["states"]), _p(s["descs"]),
                                     self.n, _p(s["colliders"]), _p(s["owners"]), len(s["colliders"]),
                                     _p(s["sources"]), len(s["sources"]), _p(s["vertices"]), len(s["vertices"]),
                                     pair_capacity, contact_capacity)
        if not self._h:
            raise ValueError("oracle refused the scene: collider owners or hull sources out of range")
        if "body_world" in s:
            L.orc_set_body_worlds(self._h, _p(s["body_world"]), len(s["body_world"]))
        L.orc_set_hull_triangles.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32]
        for source, tris in enumerate(scene.get("hull_triangles", [])):
            tris = np.ascontiguousarray(tris, np.uint32).reshape(-1, 3)
            self._keep[f"hull_triangles_{source}"] = tris
            L.orc_set_hull_triangles(self._h, source, _p(tris), len(tris))
        if "constraint_descs" in s:
            m = len(s["constraint_descs"])
            if not L.orc_set_constraints(self._h, _p(s["constraint_descs"]), _p(s["constraint_rows"]),
                                         _p(s["constraint_runtime"]), m):
                raise ValueError("oracle refused the constraints: rows out of range or a kind other than ball")

    def close(self):
        if self._h:
            lib().orc_world_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt: float) -> None:
        lib().orc_step(self._h, float(dt))

    def set_solver_guard(self, flags: int) -> None:
        """The library's solver guards (dyn_set_solver_guard), restated: 1 = the row-mass guard."""
        L = lib()
        L.orc_set_solver_guard.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        L.orc_set_solver_guard(self._h, int(flags))

    def set_ccd(self, body_id: int, enabled: bool = True) -> None:
        """World::set_ccd on the body's descriptor (dyn_set_ccd), with the wake it queues."""
        row = {int(b): r for r, b in enumerate(self.states()["body_id"])}[int(body_id)]
        L = lib()
        L.orc_set_ccd.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_set_ccd(self._h, row, 1 if enabled else 0)
        self.edit_bodies([body_id], R.body_edit(R.EDIT_WAKE))

    def edit_bodies(self, body_ids, edits: np.ndarray) -> None:
        """Queues BodyEdit records for the next step (body ids mapped to this world's rows)."""
        ids = np.asarray(body_ids, np.int64)
        row_of = {int(b): r for r, b in enumerate(self.states()["body_id"])}
        rows = np.array([row_of.get(int(i), R.NO_BODY) for i in ids], np.uint32)
        recs = np.ascontiguousarray(edits, R.BODY_EDIT)
        lib().orc_queue_edits(self._h, _p(rows), _p(recs), len(rows))

    def counters(self) -> np.ndarray:
        out = np.zeros(R.COUNTER_DEVICE_COUNT, np.uint32)
        lib().orc_counters(self._h, _p(out))
        return out

    def states(self) -> np.ndarray:
        out = np.zeros(self.n, R.BODY_STATE)
        lib().orc_states(self._h, _p(out))
        return out

    def aabbs(self) -> np.ndarray:
        n = lib().orc_aabbs(self._h, None)
        out = np.zeros(n, R.AABB)
        lib().orc_aabbs(self._h, _p(out))
        return out

    def entries(self):
        n = lib().orc_entry_keys(self._h, None, None)
        keys = np.zeros(n, np.uint32)
        infos = np.zeros(n, np.uint32)
        lib().orc_entry_keys(self._h, _p(keys), _p(infos))
        return keys, infos

    def pairs(self):
        n = lib().orc_pairs(self._h, None, None)
        major = np.zeros(n, np.uint32)
        minor = np.zeros(n, np.uint32)
        lib().orc_pairs(self._h, _p(major), _p(minor))
        return major, minor

    def contacts(self) -> np.ndarray:
        n = lib().orc_contacts(self._h, None)
        out = np.zeros(n, R.CONTACT)
        lib().orc_contacts(self._h, _p(out))
        return out

    def constraints(self) -> np.ndarray:
        n = lib().orc_constraints(self._h, None)
        out = np.zeros(n, R.CONSTRAINT_RUNTIME)
        lib().orc_constraints(self._h, _p(out))
        return out

    def joint_plan(self) -> dict:
        sizes = np.zeros(3, np.uint32)
        lib().orc_joint_plan(self._h, None, None, None, _p(sizes))
        rows = np.zeros(sizes[0], np.uint32)
        layers = np.zeros((sizes[1], 2), np.uint32)
        comps = np.zeros((sizes[2], 2), np.uint32)
        lib().orc_joint_plan(self._h, _p(rows), _p(layers), _p(comps), None)
        return {"rows": rows, "layers": layers, "components": comps}

    def query(self, queries: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """A batch of scene queries (records.QUERY) against this world's current states: the records
        with hit_base, count and overflow set, and the hit array (records.QUERY_HIT)."""
        q = np.array(queries, R.QUERY).reshape(-1)
        bound = int(np.minimum(q["max_hits"], R.QUERY_CANDIDATES).sum())
        hits = np.zeros(max(bound, 1), R.QUERY_HIT)
        L = lib()
        L.orc_query.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]
        L.orc_query(self._h, _p(q), len(q), _p(hits))
        return q, hits[:bound]

    def resting(self) -> np.ndarray:
        """The frozen contacts: first id, its generation, second id, its generation, collider a, collider b."""
        L = lib()
        L.orc_resting.restype = ctypes.c_uint32
        L.orc_resting.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        n = L.orc_resting(self._h, None)
        out = np.zeros((n, 6), np.uint32)
        if n:
            L.orc_resting(self._h, _p(out))
        return out

    def islands(self) -> np.ndarray:
        n = lib().orc_islands(self._h, None)
        out = np.zeros(n, np.uint32)
        lib().orc_islands(self._h, _p(out))
        return out


def oracle_from_world(world, dt: float, **capacity) -> OracleWorld:
    """An oracle world holding exactly the records `world` uploads to the device."""
    return OracleWorld(world.export_scene(), world.step_params(dt), **capacity)


def threads() -> int:
    """Host threads the oracle's parallel loops use."""
    return int(lib().orc_threads())


def set_threads(n: int) -> None:
    """Sets the oracle's host thread count (its results are the same for any count)."""
    lib().orc_set_threads(max(int(n), 1))


def radix_sort(major, minor=None, payload=None, major_digits=4, minor_digits=0):
    major = np.array(major, np.uint32)
    minor = np.zeros_like(major) if minor is None else np.array(minor, np.uint32)
    pay = None if payload is None else np.array(payload, np.uint32)
    lib().orc_radix_sort(_p(major), _p(minor), _p(pay), len(major), major_digits, minor_digits)
    return major, minor, pay


def config_default() -> np.ndarray:
    """PhysicsConfig::default, restated (scene.cpp)."""
    c = np.zeros(1, R.CONFIG)
    lib().orc_config_default(_p(c))
    return c


def hull_from_mesh(points, triangles=None):
    """dynamis-hull's hull() of a mesh (every point counts as referenced when triangles is None):
    the hull's vertices in the reference's order and its triangles."""
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    if triangles is None:
        idx = np.arange(len(pts), dtype=np.uint32)
        idx = np.concatenate([idx, np.full((-len(idx)) % 3, len(pts) - 1, np.uint32)])
        tris = idx.reshape(-1, 3)
    else:
        tris = np.ascontiguousarray(triangles, np.uint32).reshape(-1, 3)
    n = lib().orc_hull_from_mesh(_p(pts), len(pts), _p(tris), len(tris), None, None, 0, None)
    if n == 0:
        raise ValueError("the mesh spans no volume")
    out = np.zeros((n, 3), np.float32)
    count = ctypes.c_uint32()
    lib().orc_hull_from_mesh(_p(pts), len(pts), _p(tris), len(tris), _p(out), None, 0, ctypes.byref(count))
    faces = np.zeros((count.value, 3), np.uint32)
    lib().orc_hull_from_mesh(_p(pts), len(pts), _p(tris), len(tris), _p(out), _p(faces), count.value, None)
    return out, faces


def scene_records(bodies: np.ndarray, colliders: np.ndarray, hulls=(), worlds=None, config=None, dt: float = 1.0 / 60.0):
    """The records a world of these bodies (BODY_DESC), colliders (COLLIDER_DESC) and hull point
    sets uploads, built by the oracle's restatement of the reference's spawn path (no product code):
    a dict like World.export_scene(), with "params" = its StepParams for a step of dt."""
    L = lib()
    bodies = np.ascontiguousarray(bodies, R.BODY_DESC)
    colliders = np.ascontiguousarray(colliders, R.COLLIDER_DESC)
    pts = [np.ascontiguousarray(h, np.float32).reshape(-1, 3) for h in hulls]
    first = np.zeros(len(pts) + 1, np.uint32)
    if pts:
        first[1:] = np.cumsum([len(p) for p in pts])
    flat = np.ascontiguousarray(np.concatenate(pts) if pts else np.zeros((0, 3), np.float32))
    cfg = None if config is None else np.ascontiguousarray(config, R.CONFIG)
    handle = L.orc_scene_build(_p(cfg), _p(flat), _p(first), None, None, len(pts), _p(bodies), len(bodies),
                               _p(colliders), len(colliders))
    try:
        error = L.orc_scene_error(handle)
        if error:
            raise ValueError(f"the oracle could not build {'hull' if error < 0 else 'body'} {abs(error) - 1}")
        sizes = [ctypes.c_uint32() for _ in range(5)]
        L.orc_scene_sizes(handle, *[ctypes.byref(x) for x in sizes])
        n, dynamic, k, sources, vertices = (x.value for x in sizes)
        out = {"states": np.zeros(n, R.BODY_STATE), "descs": np.zeros(n, R.BODY_DESCRIPTOR),
               "colliders": np.zeros(k, R.COLLIDER), "owners": np.zeros(k, np.uint32),
               "sources": np.zeros(sources, R.SHAPE_SOURCE), "vertices": np.zeros((vertices, 4), np.float32),
               "dynamic": dynamic, "params": np.zeros(1, R.STEP_PARAMS)}
        L.orc_scene_export(handle, _p(out["states"]), _p(out["descs"]), _p(out["colliders"]), _p(out["owners"]),
                           _p(out["sources"]), _p(out["vertices"]))
        L.orc_scene_params(handle, float(dt), _p(out["params"]))
        if worlds is not None:
            body_world = np.asarray(worlds, np.uint32)[out["states"]["body_id"]]
            if body_world.any():
                out["body_world"] = body_world
        return out
    finally:
        L.orc_scene_free(handle)
