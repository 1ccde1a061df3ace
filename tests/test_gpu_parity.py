"""GPU step vs the CPU oracle on identical inputs, through the C ABI.

Integer products (sorted cell keys, entry infos, sorted pair lists, contact counts and features,
island ids, counters) must match exactly. Floating-point products must agree within
1e-5 relative + 1e-6 absolute (the single-step state tolerance); with IEEE single precision on
both sides and the same operand order they are expected to match bit for bit.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from dynamis_b200 import records as R
from oracle.oracle import oracle_from_world

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-5, 1e-6
DT = 1.0 / 60.0
EXACT_COUNTERS = ["ENTRIES", "IMMOVABLE_ENTRIES", "RESTING_ENTRIES", "RESTING_LEVELS", "PAIRS", "GRID_LEVELS", "IMMOVABLE_LEVELS", "CONTACTS",
                  "ISLANDS", "LIVE", "SOLVER_ROWS", "BLOCKS", "SLEPT", "WOKE", "ACTIVE", "COARSE_ACTIVE",
                  "GRID_SCALE", "GRID_EXTENT", "REFUSED_PAIRS", "REFUSED_CONTACTS", "ENTRY_FAULTS", "ARCHIVED"]


def close(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= ATOL + RTOL * np.abs(b))


def compare_step(world, oracle, step):
    gk, gi = world.debug_entries()
    ok, oi = oracle.entries()
    assert np.array_equal(gk, ok), f"step {step}: sorted cell keys differ"
    assert np.array_equal(gi, oi), f"step {step}: entry infos differ"
    gmaj, gmin = world.debug_pairs()
    omaj, omin = oracle.pairs()
    assert np.array_equal(gmaj, omaj) and np.array_equal(gmin, omin), f"step {step}: pair lists differ"
    gc, oc = world.debug_contacts(), oracle.contacts()
    assert len(gc) == len(oc), f"step {step}: contact counts differ ({len(gc)} vs {len(oc)})"
    for f in ("a", "b", "point_count", "sensor", "first_body_id", "second_body_id", "events"):
        assert np.array_equal(gc[f], oc[f]), f"step {step}: contact field {f} differs"
    for f in ("normal", "friction", "restitution", "carried_normal", "carried_tangent"):
        assert close(gc[f], oc[f]), f"step {step}: contact field {f} differs"
    mask = np.arange(4)[None, :] < oc["point_count"][:, None]
    gp, op = gc["points"][mask], oc["points"][mask]
    assert np.array_equal(gp["feature"], op["feature"]), f"step {step}: manifold features differ"
    for f in ("position", "depth", "local_a", "local_b", "accumulated_normal", "accumulated_tangent_1",
              "accumulated_tangent_2"):
        assert close(gp[f], op[f]), f"step {step}: manifold field {f} differs"
    assert np.array_equal(world.debug_islands(), oracle.islands()), f"step {step}: island ids differ"
    gm, om = world.measured(), oracle.counters()
    for name in EXACT_COUNTERS:
        assert gm[R.COUNTER[name]] == om[R.COUNTER[name]], f"step {step}: counter {name} {gm[R.COUNTER[name]]} vs {om[R.COUNTER[name]]}"
    gs, os_ = world.read_states(), oracle.states()
    for f in ("position", "orientation", "velocity", "angular_velocity", "prev_position", "prev_orientation",
              "sleep_timer"):
        assert close(gs[f], os_[f]), f"step {step}: body {f} differs"
    assert np.array_equal(gs["sleeping"], os_["sleeping"]), f"step {step}: sleep flags differ"


def run(scene, steps, dt=DT, **world_kw):
    world = World(**world_kw)
    scene.build(world)
    oracle = oracle_from_world(world, dt)
    for step in range(steps):
        world.step(dt)
        oracle.step(dt)
        world.wait()
        compare_step(world, oracle, step)
    world.close()
    return oracle


@pytest.mark.parametrize("seed", [5, 11])
def test_random_mix_matches_oracle(seed):
    run(scenes.random_mix(40, seed=seed), steps=6)


def test_falling_boxes_matches_oracle():
    run(scenes.falling_boxes(seed=0), steps=4)


def test_small_mixed_pile_matches_oracle():
    oracle = run(scenes.mixed_pile(side=6, seed=2), steps=3)
    assert oracle.counters()[R.COUNTER["PAIRS"]] > 0


def test_sphere_chain_pairs():
    oracle = run(scenes.sphere_row(16), steps=1)
    assert oracle.counters()[R.COUNTER["PAIRS"]] == 15


def test_box_tower_matches_oracle():
    run(scenes.box_tower(8), steps=5)


def test_caller_stream_gives_the_same_step():
    torch = pytest.importorskip("torch")
    scene = scenes.random_mix(40, seed=8)
    a = World()
    scene.build(a)
    b = World()
    scene.build(b)
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)  # before the first step: the scene must still be uploaded
    for _ in range(3):
        a.step(DT)
        b.step(DT)
    a.wait()
    b.wait()
    assert a.measured()[R.COUNTER["PAIRS"]] > 0
    assert np.array_equal(a.measured(), b.measured())
    assert a.read_states().tobytes() == b.read_states().tobytes()


def test_state_upload_download_round_trip():
    world = World()
    scenes.random_mix(20, seed=2).build(world)
    world.step(DT)
    states = world.read_states()
    states["velocity"] += np.float32(0.25)
    states["sleep_timer"] = np.float32(0.125)
    world.upload_states(states)
    back = world.read_states()
    assert back.tobytes() == states.tobytes()


def test_forming_pile_matches_oracle_every_step():
    """45 steps of a 1,000-body mixed pile: bodies land and rest, so penetrating hull contacts
    (EPA), warm-started impulses and sleeping all occur; every step is compared."""
    run(scenes.mixed_pile(side=10, seed=4), steps=45)
