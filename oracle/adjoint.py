"""FP64 reference gradients of the differentiable step (oracle/adjoint64.cpp through ctypes).

TEST INFRASTRUCTURE ONLY: the checker of the device adjoint (dyn_step_backward), used by tests/ and
by bench.py's check of the differentiable workload. A trajectory is recorded once with the FP32
oracle (the restated step, bit-exact with the device); each of its steps contributes its frozen
contact set (the contacts as the substeps received them, their relay sources). Over those sets the
FP64 forward of adjoint64.cpp is a smooth function of the parameters (per-row inverse mass and
inverse inertia, per-group friction, the start state), whose directional derivatives (forward mode,
exact to rounding) and central differences are the reference the device gradient is checked against.
"""
from __future__ import annotations

import ctypes

import numpy as np

from dynamis_b200 import records as R

from .oracle import _p, lib

P = ctypes.c_void_p
U32 = ctypes.c_uint32

_bound = False


def _lib():
    global _bound
    L = lib()
    if not _bound:
        L.orc_solve_contacts.restype = U32
        L.orc_solve_contacts.argtypes = [P, P, P, P]
        L.adj_forward.restype = ctypes.c_double
        L.adj_forward.argtypes = [U32, P, P, U32, P, P, P, P, P, P, P, P, P, P, U32, P, P]
        L.adj_directional.restype = None
        L.adj_directional.argtypes = [U32, P, P, U32, P, P, P, P, P, P, P, P, P, P, U32, P, U32, P, P]
        L.orc_keep_snapshots.argtypes = [P, U32]
        L.orc_step_snapshots.argtypes = [P, P, P, P, P]
        L.orc_step_decisions.restype = None
        L.orc_step_decisions.argtypes = [P, P, P, P, P]
        _bound = True
    return L


def state_vector(states: np.ndarray) -> np.ndarray:
    """BodyStateRecords as the 13 doubles per row the FP64 step takes (position, orientation xyzw,
    velocity, angular velocity)."""
    return np.concatenate([states["position"], states["orientation"], states["velocity"],
                           states["angular_velocity"]], axis=1).astype(np.float64)


class FrozenTrajectory:
    """A trajectory of the FP32 oracle, recorded step by step, as the FP64 frozen-contact problem.

    scene: the world's exported records (World.export_scene()); params: its StepParams record;
    groups: the friction group of every body row (a contact takes its first body's group, or its
    second's when the first is static); target: the loss's target positions (rows x 3)."""

    def __init__(self, oracle_world, scene: dict, params: np.ndarray, steps: int, dt: float, groups: np.ndarray,
                 start: np.ndarray | None = None):
        L = _lib()
        self.n = len(scene["states"])
        self.dynamic_count = int(np.atleast_1d(params)["dynamic_count"][0])
        # the state the first step's solve starts from (the caller passes it when queued edits change it)
        self.start = oracle_world.states() if start is None else start
        self.counts, self.cint, self.cdouble, self.cpoints, self.sources = [], [], [], [], []
        self.contact_friction = []
        self.decisions = []
        self.follow_decisions = False  # True: branches as the recorded FP32 run took them
        self.along_record = False      # True: derivatives along the recorded FP32 run's values (with its branches)
        descs = scene["descs"]
        dyn_rows = (descs["inverse_mass"] > 0) & ((descs["flags"] & 1) == 0) & (self.start["sleeping"] == 0)
        dyn_rows &= np.arange(self.n) < self.dynamic_count
        self.dynamic = dyn_rows
        L.orc_keep_snapshots(oracle_world._h, 1)
        pp = np.atleast_1d(params)
        K, I, PI = int(pp["substeps"][0]), int(pp["solve_iterations"][0]), int(pp["position_iterations"][0])
        self.snapshots = []
        for step in range(steps):
            oracle_world.step(dt)
            c = L.orc_solve_contacts(oracle_world._h, None, None, None)
            rec = np.zeros(c, R.CONTACT)
            targets = np.zeros(4 * c, np.float32)
            src = np.zeros(4 * c, np.int32)
            L.orc_solve_contacts(oracle_world._h, _p(rec), _p(targets), _p(src))
            owners = scene["owners"]
            a = owners[rec["a"]].astype(np.int64)
            b = owners[rec["b"]].astype(np.int64)
            group = np.where(self.dynamic[a], groups[a], groups[b])
            ints = np.stack([a, b, rec["point_count"], group, ((rec["point_count"] > 0) & (rec["sensor"] == 0))],
                            axis=1).astype(np.int32)
            dbl = np.concatenate([rec["normal"], rec["restitution"][:, None], rec["rolling_friction"][:, None],
                                  rec["spin_friction"][:, None], rec["relaxation"][:, None],
                                  rec["damping_ratio"][:, None]], axis=1).astype(np.float64)
            pts = rec["points"]
            acc = np.stack([pts["accumulated_normal"], pts["accumulated_tangent_1"], pts["accumulated_tangent_2"]],
                           axis=2)
            per_point = np.concatenate([pts["local_a"], pts["local_b"], pts["depth"][:, :, None], pts["position"], acc,
                                        np.zeros((c, 4, 3), np.float32)], axis=2).astype(np.float64)
            if step == 0:
                src[:] = -1  # the first step's impulses are given (relayed from before the trajectory)
            self.counts.append(c)
            self.cint.append(ints)
            self.cdouble.append(dbl)
            self.cpoints.append(per_point.reshape(c, 64))
            self.sources.append(src.reshape(c, 4))
            self.contact_friction.append(rec["friction"])
            K = int(np.atleast_1d(params)["substeps"][0])
            I = int(np.atleast_1d(params)["solve_iterations"][0])
            PI = int(np.atleast_1d(params)["position_iterations"][0])
            solve = np.zeros(K * I * 4 * c, np.uint8)
            position = np.zeros(K * PI * 4 * c, np.uint8)
            integrate = np.zeros(K * self.n, np.uint8)
            target_flags = np.zeros(4 * c, np.uint8)
            L.orc_step_decisions(oracle_world._h, _p(solve), _p(position), _p(integrate), _p(target_flags))
            self.decisions.append(np.concatenate([solve, position, integrate, target_flags]))
            snaps = [np.zeros(K * self.n * 13, np.float32), np.zeros(K * I * self.n * 6, np.float32),
                     np.zeros(K * I * c * 12, np.float32), np.zeros(K * PI * self.n * 3, np.float32)]
            L.orc_step_snapshots(oracle_world._h, *[_p(a) for a in snaps])
            self.snapshots.append(np.concatenate(snaps))
        self.final = oracle_world.states()
        L.orc_keep_snapshots(oracle_world._h, 0)
        self.decisions = np.ascontiguousarray(np.concatenate(self.decisions) if self.decisions else np.zeros(0, np.uint8))
        self.snapshots = np.ascontiguousarray(np.concatenate(self.snapshots) if self.snapshots else np.zeros(0, np.float32))
        self.final_record = np.ascontiguousarray(state_vector(self.final).astype(np.float32))
        self.counts = np.array(self.counts, np.uint32)
        self.cint = np.ascontiguousarray(np.concatenate(self.cint) if self.cint else np.zeros((0, 5), np.int32))
        self.cdouble = np.ascontiguousarray(np.concatenate(self.cdouble) if self.cdouble else np.zeros((0, 8)))
        self.cpoints = np.ascontiguousarray(np.concatenate(self.cpoints) if self.cpoints else np.zeros((0, 64)))
        self.sources = np.ascontiguousarray(np.concatenate(self.sources) if self.sources else np.zeros((0, 4), np.int32))
        self.groups = int(groups.max()) + 1
        self.contact_groups = self.cint[:, 3]
        com = descs["com"].astype(np.float64)
        inertia = descs["inertia"].astype(np.float64)
        self.bodies = np.zeros((self.n, 20), np.float64)
        self.bodies[:, 0] = descs["inverse_mass"]
        self.bodies[:, 1:7] = descs["inverse_inertia"]
        self.bodies[:, 7:10] = com
        self.bodies[:, 10] = descs["gravity_scale"]
        self.bodies[:, 11] = descs["linear_damping"]
        self.bodies[:, 12] = descs["angular_damping"]
        self.bodies[:, 13:19] = inertia
        self.bodies[:, 19] = self.dynamic
        p = np.atleast_1d(params)
        self.params = np.array([p["dt"][0], *p["gravity"][0][:3], p["slop"][0], p["relaxation"][0],
                                p["restitution_threshold"][0], p["max_velocity"][0], p["max_angular_velocity"][0],
                                p["substeps"][0], p["solve_iterations"][0], p["position_iterations"][0]], np.float64)
        self.target = np.zeros((self.n, 3), np.float64)

    @property
    def dim(self) -> int:
        """Length of the parameter vector [inverse_mass, inverse_inertia (6), friction (groups), state (13)]."""
        return 20 * self.n + self.groups

    def _args(self, inverse_mass, inverse_inertia, friction, state):
        bodies = self.bodies.copy()
        bodies[:, 0] = inverse_mass
        bodies[:, 1:7] = inverse_inertia
        self._keep = (np.ascontiguousarray(bodies), np.ascontiguousarray(self.target, np.float64),
                      np.ascontiguousarray(friction, np.float64), np.ascontiguousarray(state, np.float64))
        b, t, f, s = self._keep
        dec = _p(self.decisions) if (self.follow_decisions or self.along_record) else None
        snaps = _p(self.snapshots) if self.along_record else None
        fin = _p(self.final_record) if self.along_record else None
        return (len(self.bodies), _p(b), _p(self.params), len(self.counts), _p(self.counts), _p(self.cint),
                _p(self.cdouble), _p(self.cpoints), _p(self.sources), _p(t), dec, snaps, fin, _p(f), len(f), _p(s))

    def forward(self, inverse_mass, inverse_inertia, friction, state):
        """The FP64 loss and final state (rows x 13) of the frozen-contact trajectory."""
        out = np.zeros((self.n, 13), np.float64)
        loss = _lib().adj_forward(*self._args(inverse_mass, inverse_inertia, friction, state), _p(out))
        return loss, out

    def directional(self, inverse_mass, inverse_inertia, friction, state, tangents: np.ndarray) -> np.ndarray:
        """d loss / d t for every row t of `tangents` (k x dim), forward mode in FP64."""
        tangents = np.ascontiguousarray(tangents, np.float64)
        out = np.zeros(len(tangents), np.float64)
        _lib().adj_directional(*self._args(inverse_mass, inverse_inertia, friction, state), len(tangents),
                               _p(tangents), _p(out))
        return out

    # parameter-vector offsets
    def inverse_mass_slot(self, row: int) -> int:
        return row

    def inverse_inertia_slot(self, row: int, k: int) -> int:
        return self.n + 6 * row + k

    def friction_slot(self, group: int) -> int:
        return 7 * self.n + group

    def state_slot(self, row: int, k: int) -> int:
        return 7 * self.n + self.groups + 13 * row + k
