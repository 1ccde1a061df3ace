"""Pins the oracle (the CPU restatement of the step) before it is trusted as the checker.

The reference holds no golden state vectors; its tests pin behaviours, restated here on the oracle:
  * key_words table, stable payload sort        crates/dynamis-sort/tests/gpu.rs:192-249, 313-320
  * one pair for two overlapping spheres at any offset, 15 pairs for a 16-sphere chain, one pair
    per body on a wide floor                      crates/dynamis-world/tests/suite/broadphase.rs:297-352
  * free fall against the symplectic closed form  dynamics.rs:11-31 with common.rs:58-62
  * a two-sphere stack rests at its heights       dynamics.rs:164-175
  * a 16-box tower holds its spacing              dynamics.rs:177-213
  * a dropped box settles within margin + slop    dynamics.rs:215-240
  * bit-for-bit determinism of two runs           determinism.rs:61-89
plus the restatement's own math (Cephes sin/cos/atan2 against libm) and the grid broadphase
against a brute-force AABB overlap test.
"""
import numpy as np
import pytest

from dynamis_b200 import World, scenes
from dynamis_b200 import records as R
from oracle import oracle as O

DT = 1.0 / 60.0


def static_config():
    return {"gravity": (0.0, 0.0, 0.0), "damping": 0.0, "angular_damping": 0.0}


def gravity_config():
    return {"damping": 0.0, "angular_damping": 0.0}


def make(bodies, config=None):
    """bodies: list of dicts (shape, position, mass or density, collider fields)."""
    w = World(**(config or {}))
    n = len(bodies)
    b = R.body_defaults(n)
    c = R.collider_defaults(n)
    for i, spec in enumerate(bodies):
        spec = dict(spec)
        b["position"][i] = spec.pop("position", (0, 0, 0))
        for key in ("mass", "density", "velocity", "angular_velocity", "orientation"):
            if key in spec:
                b[key][i] = spec.pop(key)
        for key, value in spec.items():
            c[key][i] = value
    ids = w.spawn(b, c)
    return w, ids


def oracle_of(world, dt=DT):
    return O.oracle_from_world(world, dt)


def state_of(oracle, world, body_id):
    s = oracle.states()
    return s[s["body_id"] == body_id][0]


# ---- math ----

def test_cephes_sin_cos_within_two_ulp():
    L = O.lib()
    xs = np.concatenate([np.linspace(-20, 20, 4001), np.linspace(-1e-3, 1e-3, 101), [0.5 * np.pi, np.pi, 3.0]])
    for x in xs.astype(np.float32):
        for fn, ref in ((L.orc_sin, np.sin), (L.orc_cos, np.cos)):
            got = np.float32(fn(float(x)))
            want = ref(np.float64(x))
            ulp = np.spacing(np.float32(abs(want))) if want != 0 else np.float32(1e-38)
            assert abs(np.float64(got) - want) <= max(2 * ulp, 2e-8), (fn, x, got, want)


def test_cephes_atan2_quadrants():
    L = O.lib()
    rng = np.random.default_rng(0)
    pts = rng.normal(size=(2000, 2)).astype(np.float32)
    for y, x in pts:
        got = L.orc_atan2(float(y), float(x))
        assert abs(got - np.arctan2(np.float64(y), np.float64(x))) < 4e-7
    assert L.orc_atan2(0.0, -1.0) == np.float32(np.pi)
    assert L.orc_atan2(1.0, 0.0) == np.float32(np.pi / 2)


# ---- sort ----

def test_key_words_cover_the_index_space():
    L = O.lib()
    assert [L.orc_key_words(n) for n in (1, 256, 257, 1 << 16, 1 << 24, 0xFFFFFFFF)] == [1, 1, 2, 2, 3, 4]


def test_radix_sort_is_stable_and_carries_the_payload():
    rng = np.random.default_rng(1)
    keys = rng.integers(0, 64, size=5000, dtype=np.uint32)
    pay = np.arange(5000, dtype=np.uint32)
    major, _, carried = O.radix_sort(keys, payload=pay, major_digits=4)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(major, keys[order]) and np.array_equal(carried, pay[order])


def test_radix_sort_two_words():
    rng = np.random.default_rng(2)
    major = rng.integers(0, 1 << 18, size=300000, dtype=np.uint32)
    minor = rng.integers(0, 1 << 18, size=300000, dtype=np.uint32)
    smaj, smin, _ = O.radix_sort(major, minor, major_digits=3, minor_digits=3)
    order = np.lexsort((minor, major))
    assert np.array_equal(smaj, major[order]) and np.array_equal(smin, minor[order])


# ---- broadphase ----

@pytest.mark.parametrize("offset", [0.05, 0.2, 0.35, 0.5, 0.65])
def test_a_collider_pair_enters_the_candidate_stream_exactly_once(offset):
    w, _ = make([dict(shape=R.SHAPE_SPHERE, radius=0.35, mass=0.0),
                 dict(shape=R.SHAPE_SPHERE, radius=0.35, position=(offset, 0, 0))], static_config())
    o = oracle_of(w)
    o.step(DT)
    c = o.counters()
    assert c[R.COUNTER["PAIRS"]] == 1 and c[R.COUNTER["REFUSED_PAIRS"]] == 0


def test_a_chain_emits_one_pair_per_touching_neighbour():
    w, _ = make([dict(shape=R.SHAPE_SPHERE, radius=0.4, position=(i * 0.5, 0, 0)) for i in range(16)],
                static_config())
    o = oracle_of(w)
    o.step(DT)
    assert o.counters()[R.COUNTER["PAIRS"]] == 15


def test_a_coarse_collider_emits_one_pair_per_covered_collider():
    specs = [dict(shape=R.SHAPE_CUBOID, half_extents=(30.0, 0.5, 30.0), mass=0.0, position=(0, -0.5, 0))]
    for i in range(64):
        specs.append(dict(shape=R.SHAPE_SPHERE, radius=0.4, position=((i % 8) - 3.5, 0.4, (i // 8) - 3.5)))
    w, _ = make(specs, static_config())
    o = oracle_of(w)
    o.step(DT)
    assert o.counters()[R.COUNTER["PAIRS"]] == 64


def brute_force_pairs(oracle, world):
    scene = world.export_scene()
    aabb = oracle.aabbs()
    owners = scene["owners"]
    descs = scene["descs"]
    moves = (descs["inverse_mass"] > 0) | ((descs["flags"] & 1) != 0)
    states = scene["states"]
    awake = moves & (states["sleeping"] == 0)
    out = set()
    k = len(aabb)
    for a in range(k):
        for b in range(a + 1, k):
            ra, rb = owners[a], owners[b]
            if ra == rb or not (moves[ra] or moves[rb]) or not (awake[ra] or awake[rb]):
                continue
            if np.all(aabb["min"][a] <= aabb["max"][b]) and np.all(aabb["min"][b] <= aabb["max"][a]):
                out.add((a, b))
    return out


@pytest.mark.parametrize("seed", [3, 9])
def test_grid_broadphase_finds_exactly_the_overlapping_pairs(seed):
    w = World()
    scenes.random_mix(60, seed=seed).build(w)
    o = oracle_of(w)
    o.step(DT)
    major, minor = o.pairs()
    got = list(zip(major.tolist(), minor.tolist()))
    assert len(got) == len(set(got)), "a pair was emitted twice"
    assert got == sorted(got), "pairs are not sorted by (major, minor)"
    assert set(got) == brute_force_pairs(o, w)


# ---- dynamics ----

def symplectic_fall(gravity, frames, initial_speed, substeps, dt=DT):
    step = np.float32(dt / substeps)
    count = np.float32(frames * substeps)
    return initial_speed * step * count - 0.5 * gravity * step * step * count * (count + 1.0)


def test_free_fall_matches_closed_form():
    w, ids = make([dict(shape=R.SHAPE_SPHERE, radius=0.1, position=(0, 10, 0), mass=1.0)], gravity_config())
    o = oracle_of(w)
    for _ in range(30):
        o.step(DT)
    s = state_of(o, w, ids[0])
    assert abs(s["position"][1] - (10.0 + symplectic_fall(9.81, 30, 0.0, 2))) < 1e-3
    assert abs(s["velocity"][1] - (-9.81 * DT * 30)) < 1e-3


def test_stacked_bodies_do_not_collapse():
    w, ids = make([dict(shape=R.SHAPE_SPHERE, radius=1.0, mass=0.0),
                   dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 1.5, 0)),
                   dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(0, 2.5, 0))], gravity_config())
    o = oracle_of(w)
    for _ in range(120):
        o.step(DT)
        if o.counters()[R.COUNTER["ACTIVE"]] == 0:
            break
    lower, upper = state_of(o, w, ids[1]), state_of(o, w, ids[2])
    assert 1.4 < lower["position"][1] < 1.52
    assert 2.4 < upper["position"][1] < 2.6


def test_a_resting_tower_holds_its_spacing():
    specs = [dict(shape=R.SHAPE_CUBOID, half_extents=(40.0, 0.5, 40.0), mass=0.0, position=(0, -0.5, 0))]
    for level in range(16):
        specs.append(dict(shape=R.SHAPE_CUBOID, half_extents=(0.5, 0.5, 0.5), position=(0, 0.5 + level * 1.0005, 0),
                          friction=0.7, restitution=0.0))
    w, ids = make(specs)
    o = oracle_of(w)
    for _ in range(240):
        o.step(DT)
    s = o.states()
    for level in range(16):
        st = s[s["body_id"] == ids[level + 1]][0]
        assert abs(st["position"][1] - (0.5 + level)) <= 0.02 + level * 0.005, (level, st["position"])
        assert abs(st["position"][0]) < 0.2 and abs(st["position"][2]) < 0.2


def test_a_dropped_body_settles_within_the_contact_margin():
    w, ids = make([dict(shape=R.SHAPE_CUBOID, half_extents=(40.0, 0.5, 40.0), mass=0.0, position=(0, -0.5, 0)),
                   dict(shape=R.SHAPE_CUBOID, half_extents=(0.5, 0.5, 0.5), position=(0, 2.5, 0), friction=0.7)])
    o = oracle_of(w)
    for _ in range(240):
        o.step(DT)
    overlap = 0.5 - state_of(o, w, ids[1])["position"][1]
    assert overlap <= 0.02 + 0.005


def test_boxes_come_to_rest_on_a_plane_and_sleep():
    w = World()
    scenes.box_tower(3).build(w)
    o = oracle_of(w)
    slept = 0
    for _ in range(200):
        o.step(DT)
        slept += int(o.counters()[R.COUNTER["SLEPT"]])
    s = o.states()
    assert slept >= 3 and np.all(s["sleeping"][:3] == 1)
    assert np.allclose(s["position"][:3, 1], [0.5, 1.5, 2.5], atol=0.03)


def test_two_runs_are_bit_identical():
    def run():
        w = World()
        scenes.random_mix(30, seed=4).build(w)
        o = oracle_of(w)
        for _ in range(20):
            o.step(DT)
        return o.states()

    a, b = run(), run()
    assert a.tobytes() == b.tobytes()


def test_islands_are_minimum_rows_of_touching_groups():
    specs = [dict(shape=R.SHAPE_SPHERE, radius=0.5, position=(x, 0, 0)) for x in (0.0, 0.9, 1.8, 10.0, 10.9)]
    w, ids = make(specs, static_config())
    o = oracle_of(w)
    o.step(DT)
    assert list(o.islands()) == [0, 0, 0, 3, 3]
    assert o.counters()[R.COUNTER["ISLANDS"]] == 2
