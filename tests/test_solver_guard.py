"""The row-mass guard (dyn_set_solver_guard, DYN_SOLVER_GUARD_ROW_MASS), on the CPU oracle.

The reference solves a contact's points together, each against its manifold row mass D_j = sum_k
A_jk (solver_contact_block.wgsl:14-29), A being the points' coupling matrix. That Jacobi iteration
converges only while the eigenvalues of D^-1 A stay below 2; where a point's arm opposes the others'
they do not, and the reference's own algorithm pumps energy into the pile. These tests pin:

* the divergence itself, on a three-point box-on-ground manifold taken from the 4,096-body mixed pile
  (step 29, the box that left at 265 m/s): the iteration matrix I - D^-1 A has an eigenvalue of -2.01,
  and the guard's bound rejects the block; count x A_jj gives a spectral radius below 1;
* the reference's algorithm (the oracle, guard off) on the 1,000-body mixed pile: within 90 steps
  the total energy rises above its start (to 1.55 x) and a body outruns free fall from the top by
  a factor of six;
* the guard on the same pile: energy never above its start, no body faster than free fall;
* the guard leaves converging blocks alone: on a tower of cubes resting face to face (four-point
  manifolds whose normalised coupling eigenvalues stay at 1.5 or below), 60 guarded steps are
  bit-identical to the reference's. (The falling boxes are not such a scene: a cube that lands on
  three points can reach 2.1 there, where the reference's iteration diverges.)
"""
import numpy as np
import pytest

from dynamis_b200 import DynamisError, World, diagnostics, scenes
from dynamis_b200 import records as R
from oracle.oracle import OracleWorld

DT = 1.0 / 60.0

# box 3328 of mixed_pile(side=16, seed=1) at the start of step 29: centre of mass, orientation
# (x, y, z, w), inverse mass, body-frame inverse inertia diagonal, the three manifold points and the
# normal (from the box to the ground)
BOX_COM = np.array([7.1919, 0.2675, -9.7807])
BOX_Q = np.array([-0.7279, 0.685, -0.0008, -0.0321])
BOX_IM = 0.0047963206
BOX_II = np.array([0.056188457, 0.052577533, 0.124118164])
POINTS = np.array([[6.9673, -0.0126, -10.2128], [7.0062, 0.0092, -9.305], [7.4095, 0.0006, -10.2331]])
NORMAL = np.array([0.0, -1.0, 0.0])


def rotation(q):
    x, y, z, w = q / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def test_the_reference_row_masses_diverge_on_a_landing_box():
    r = rotation(BOX_Q)
    inv_inertia = r @ np.diag(BOX_II) @ r.T
    arms = np.cross(POINTS - BOX_COM, NORMAL)
    a = BOX_IM + arms @ inv_inertia @ arms.T  # the ground is static: its terms vanish
    d = a.sum(axis=1)  # manifold_row_mass
    assert np.all(d > 0)
    iteration = np.eye(3) - np.diag(1.0 / d) @ a
    assert np.min(np.linalg.eigvals(iteration).real) < -2.0  # |lambda| > 1: the impulses grow
    normalised = a / np.sqrt(np.outer(d, d))
    assert np.linalg.eigvalsh(normalised).max() > 1.9  # the guard rejects the block
    fallback = np.eye(3) - np.diag(1.0 / (3 * np.diag(a))) @ a
    assert np.max(np.abs(np.linalg.eigvals(fallback))) < 1.0


def pile_run(guard: int, side: int = 10, steps: int = 90):
    world = World()
    scenes.mixed_pile(side=side, seed=1).build(world)
    exported = world.export_scene()
    oracle = OracleWorld(exported, world.step_params(DT))
    oracle.set_solver_guard(guard)
    states = oracle.states()
    start = diagnostics.energy(states, exported["descs"], (0.0, -9.81, 0.0))["total"]
    bound = float(np.sqrt(2 * 9.81 * states["position"][:, 1].max()))
    ratio, speed = 0.0, 0.0
    for _ in range(steps):
        oracle.step(DT)
        states = oracle.states()
        ratio = max(ratio, diagnostics.energy(states, exported["descs"], (0.0, -9.81, 0.0))["total"] / start)
        speed = max(speed, float(np.linalg.norm(states["velocity"].astype(np.float64), axis=1).max()))
    oracle.close()
    world.close()
    return ratio, speed, bound


def test_the_reference_solver_pumps_energy_into_the_mixed_pile():
    ratio, speed, bound = pile_run(guard=0)
    assert ratio > 1.2, ratio  # a passive system gains energy: measured 1.55 x its start
    assert speed > 3.0 * bound, (speed, bound)  # measured 97 m/s against a 16 m/s free-fall bound


def test_the_row_mass_guard_keeps_the_mixed_pile_within_bounds():
    ratio, speed, bound = pile_run(guard=1)
    assert ratio <= 1.0 + 1e-6, ratio
    assert speed <= bound, (speed, bound)


def test_the_guard_leaves_converging_blocks_alone():
    world = World()
    scenes.tower_world(seed=3, levels=8, footprint=4, gap=0.0, heading=0.0).build(world)
    exported = world.export_scene()
    plain = OracleWorld(exported, world.step_params(DT))
    guarded = OracleWorld(exported, world.step_params(DT))
    guarded.set_solver_guard(1)
    for _ in range(60):
        plain.step(DT)
        guarded.step(DT)
    assert plain.states().tobytes() == guarded.states().tobytes()
    plain.close()
    guarded.close()
    world.close()


def test_the_guard_refuses_unknown_flags_and_the_adjoint_refuses_a_guarded_world():
    world = World(sleep_time=np.inf)
    scenes.tower_world(seed=3).build(world)
    with pytest.raises(DynamisError):
        world.set_solver_guard(2)
    world.set_solver_guard(R.SOLVER_GUARD_ROW_MASS)
    with pytest.raises(DynamisError):
        world.tape_begin(10)
    world.close()
