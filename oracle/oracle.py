"""ctypes wrapper of the oracle library (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker used by tests/ and bench.py's cpu_baseline leg. It runs the
CPU restatement of the Dynamis step (oracle.cpp) on records exported from a dynamis_b200 World.
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
