"""The row-mass guard on the GPU (dyn_set_solver_guard, DYN_SOLVER_GUARD_ROW_MASS).

* Parity: the 1,000-body mixed pile, guarded on both sides, against the oracle every step for 90
  steps; the pile lands in that time and the guard replaces the row masses of the blocks where the
  reference's iteration diverges, so every product still matches (test_gpu_parity.compare_step).
* The 262,144-body mixed pile, guarded, after the benchmark's 125 setup and warm-up steps: total
  energy not above its start and no body faster than free fall from the lattice's top (the
  reference's solver fails both there: the bench reports it under setup_checks).
"""
import numpy as np
import pytest

from dynamis_b200 import World, diagnostics, scenes
from dynamis_b200 import records as R
from oracle.oracle import oracle_from_world
from test_gpu_parity import DT, compare_step

pytestmark = pytest.mark.gpu


def test_a_guarded_pile_matches_the_guarded_oracle_every_step():
    world = World()
    scenes.mixed_pile(side=10, seed=1).build(world)
    world.set_solver_guard(R.SOLVER_GUARD_ROW_MASS)
    oracle = oracle_from_world(world, DT)
    oracle.set_solver_guard(R.SOLVER_GUARD_ROW_MASS)
    for step in range(90):
        world.step(DT)
        oracle.step(DT)
        world.wait()
        compare_step(world, oracle, step)
    oracle.close()
    world.close()


def test_the_guarded_benchmark_pile_stays_within_the_long_run_bounds():
    world = World()
    scenes.WORKLOADS["mixed_pile_262144"]().build(world)
    world.set_solver_guard(R.SOLVER_GUARD_ROW_MASS)
    before = diagnostics.summary(world, DT, stepped=False)["energy"]["total"]
    top = float(world.read_states()["position"][:, 1].max())
    for _ in range(125):
        world.step(DT)
    after = diagnostics.summary(world, DT)
    speed = np.linalg.norm(world.read_states()["velocity"].astype(np.float64), axis=1)
    assert np.all(np.isfinite(speed))
    assert after["energy"]["total"] <= before * (1.0 + 1e-6), (after["energy"], before)
    assert speed.max() <= np.sqrt(2.0 * 9.81 * top), speed.max()
    world.close()
