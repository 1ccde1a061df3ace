"""The oracle against the committed golden fixtures (tests/golden/, written by make_golden.py).

sort_known_answers.json holds the known-answer cases of the reference's own radix sort tests
(crates/dynamis-sort/tests/gpu.rs:192-320); step_random_mix_24.npz is the oracle's own output for
three steps of a seeded scene, kept so that any later change to the oracle shows up here.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from dynamis_b200 import records as R
from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
DT = 1.0 / 60.0


def known_answers() -> dict:
    return json.loads((GOLDEN / "sort_known_answers.json").read_text())


def xorshift_keys(length: int, salt: int) -> np.ndarray:
    """Marsaglia's xorshift32 (13, 17, 5) from the seed 0x9E3779B9 ^ salt, the reference test's key source."""
    state = (0x9E3779B9 ^ salt) & 0xFFFFFFFF
    out = np.empty(length, np.uint32)
    for i in range(length):
        state ^= (state << 13) & 0xFFFFFFFF
        state ^= state >> 17
        state ^= (state << 5) & 0xFFFFFFFF
        out[i] = state
    return out


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()


def test_oracle_sort_ten_keys():
    case = known_answers()["ten_keys"]
    keys = np.array(case["keys"], np.uint32)
    major, _, payload = O.radix_sort(keys, payload=np.arange(len(keys), dtype=np.uint32),
                                     major_digits=case["major_digits"])
    assert major.tolist() == case["sorted"] and payload.tolist() == case["payload"]


def test_oracle_sort_major_above_minor():
    case = known_answers()["major_above_minor"]
    major, minor, payload = O.radix_sort(case["major"], case["minor"], np.arange(len(case["major"]), dtype=np.uint32),
                                         case["major_digits"], case["minor_digits"])
    assert major.tolist() == case["sorted_major"]
    assert minor.tolist() == case["sorted_minor"]
    assert payload.tolist() == case["payload"]


def test_oracle_sort_wide_two_word_keys():
    case = known_answers()["wide_two_word"]
    major = xorshift_keys(case["length"], case["major_salt"])
    minor = xorshift_keys(case["length"], case["minor_salt"])
    assert digest(major) == case["input_major_sha256"] and digest(minor) == case["input_minor_sha256"]
    smaj, smin, pay = O.radix_sort(major, minor, np.arange(case["length"], dtype=np.uint32),
                                   case["major_digits"], case["minor_digits"])
    assert digest(smaj) == case["sorted_major_sha256"]
    assert digest(smin) == case["sorted_minor_sha256"]
    assert digest(pay) == case["payload_sha256"]


def test_oracle_key_words_table():
    for n, words in known_answers()["key_words"]:
        assert O.lib().orc_key_words(n) == words


@pytest.fixture(scope="module")
def step_golden():
    return np.load(GOLDEN / "step_random_mix_24.npz")


def test_oracle_reproduces_the_step_fixture(step_golden):
    from dynamis_b200 import World, scenes

    world = World()
    scenes.random_mix(24, seed=5).build(world)
    oracle = O.oracle_from_world(world, DT)
    for s in range(3):
        oracle.step(DT)
        keys, infos = oracle.entries()
        major, minor = oracle.pairs()
        assert np.array_equal(keys, step_golden[f"s{s}_keys"]), f"step {s}: cell keys"
        assert np.array_equal(infos, step_golden[f"s{s}_infos"]), f"step {s}: entry infos"
        assert np.array_equal(major, step_golden[f"s{s}_pair_major"]), f"step {s}: pairs"
        assert np.array_equal(minor, step_golden[f"s{s}_pair_minor"]), f"step {s}: pairs"
        assert oracle.contacts().tobytes() == step_golden[f"s{s}_contacts"].tobytes(), f"step {s}: contacts"
        assert np.array_equal(oracle.islands(), step_golden[f"s{s}_islands"]), f"step {s}: islands"
        assert oracle.states().tobytes() == step_golden[f"s{s}_states"].tobytes(), f"step {s}: states"
        assert np.array_equal(oracle.counters(), step_golden[f"s{s}_counters"]), f"step {s}: counters"
    oracle.close()
    world.close()


def test_the_oracle_steps_alike_on_one_thread_and_on_many():
    """The oracle's parallel loops join their results in index order and sum integers only, so a
    step is bit-identical for any thread count."""
    from dynamis_b200 import World, scenes

    default = O.threads()
    results = []
    try:
        for n in (1, 4):
            O.set_threads(n)
            w = World()
            scenes.mixed_pile(side=6, seed=2).build(w)
            o = O.oracle_from_world(w, 1.0 / 60.0)
            for _ in range(25):
                o.step(1.0 / 60.0)
            results.append((o.states(), o.contacts(), o.counters()))
            o.close()
            w.close()
    finally:
        O.set_threads(default)
    (s1, c1, k1), (s4, c4, k4) = results
    assert k1[R.COUNTER["CONTACTS"]] > 0
    assert s1.tobytes() == s4.tobytes() and c1.tobytes() == c4.tobytes() and np.array_equal(k1, k4)
