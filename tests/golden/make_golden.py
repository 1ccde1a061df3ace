"""Writes the golden fixtures under tests/golden/. Run from the repository root:

    python tests/golden/make_golden.py

sort_known_answers.json -- the known-answer cases of the reference's radix sort tests
(crates/dynamis-sort/tests/gpu.rs): the ten-key stable sort with a counting payload (:192-212),
the 300,000-element two-word sort over xorshift32 keys (:214-250), the major-above-minor case of
64 keys (:252-275) and the key_words table (:313-320). Inputs are the ones those tests build;
expected outputs come from the definition of a stable lexicographic sort (Python's sorted /
numpy's stable lexsort), not from any code in this repository. The 300,000-element case is stored
as SHA-256 digests of the inputs and of the three sorted arrays, plus the payload's first and
last entries.

step_random_mix_24.npz -- a regression fixture produced by the oracle (oracle/oracle.cpp): three
steps of the seeded 24-body random mix, with the sorted cell keys, entry infos, sorted pairs,
contacts, island ids, counters and body states after each step, as raw record bytes. It pins the
oracle (and, in the GPU tests, the device) against later changes; it is not an output of the
reference, which cannot run here.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
DT = 1.0 / 60.0


def xorshift_keys(length: int, salt: int) -> np.ndarray:
    """Marsaglia's xorshift32 (13, 17, 5) from the seed 0x9E3779B9 ^ salt, as the reference test does."""
    state = (0x9E3779B9 ^ salt) & 0xFFFFFFFF
    out = np.empty(length, np.uint32)
    for i in range(length):
        state ^= (state << 13) & 0xFFFFFFFF
        state ^= state >> 17
        state ^= (state << 5) & 0xFFFFFFFF
        out[i] = state
    return out


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()


def sort_cases() -> dict:
    ten = [3, 5, 1, 0, 7, 2, 2, 9, 4, 6]
    ten_sorted = sorted((k, i) for i, k in enumerate(ten))
    n = 64
    major64 = [i % 4 for i in range(n)]
    minor64 = [(i * 5) % 8 for i in range(n)]
    sorted64 = sorted((major64[i], minor64[i], i) for i in range(n))
    wide = 300_000
    major = xorshift_keys(wide, 1)
    minor = xorshift_keys(wide, 2)
    order = np.lexsort((minor, major))  # stable: equal (major, minor) keep their input order
    return {
        "ten_keys": {"keys": ten, "major_digits": 1, "minor_digits": 0,
                     "sorted": [k for k, _ in ten_sorted], "payload": [i for _, i in ten_sorted]},
        "major_above_minor": {"major": major64, "minor": minor64, "major_digits": 1, "minor_digits": 1,
                              "sorted_major": [m for m, _, _ in sorted64], "sorted_minor": [m for _, m, _ in sorted64],
                              "payload": [i for _, _, i in sorted64]},
        "wide_two_word": {"length": wide, "major_salt": 1, "minor_salt": 2, "major_digits": 4, "minor_digits": 4,
                          "input_major_sha256": digest(major), "input_minor_sha256": digest(minor),
                          "sorted_major_sha256": digest(major[order]), "sorted_minor_sha256": digest(minor[order]),
                          "payload_sha256": digest(order.astype(np.uint32)),
                          "payload_head": order[:16].tolist(), "payload_tail": order[-16:].tolist()},
        "key_words": [[1, 1], [256, 1], [257, 2], [1 << 16, 2], [1 << 24, 3], [0xFFFFFFFF, 4]],
    }


def step_fixture() -> dict:
    sys.path.insert(0, str(ROOT))
    from dynamis_b200 import World, scenes
    from oracle.oracle import oracle_from_world

    world = World()
    scenes.random_mix(24, seed=5).build(world)
    oracle = oracle_from_world(world, DT)
    out = {}
    for step in range(3):
        oracle.step(DT)
        keys, infos = oracle.entries()
        major, minor = oracle.pairs()
        out[f"s{step}_keys"] = keys
        out[f"s{step}_infos"] = infos
        out[f"s{step}_pair_major"] = major
        out[f"s{step}_pair_minor"] = minor
        out[f"s{step}_contacts"] = np.frombuffer(oracle.contacts().tobytes(), np.uint8)
        out[f"s{step}_islands"] = oracle.islands()
        out[f"s{step}_states"] = np.frombuffer(oracle.states().tobytes(), np.uint8)
        out[f"s{step}_counters"] = oracle.counters()
    oracle.close()
    world.close()
    return out


def main() -> None:
    (HERE / "sort_known_answers.json").write_text(json.dumps(sort_cases(), indent=1) + "\n")
    np.savez_compressed(HERE / "step_random_mix_24.npz", **step_fixture())
    print("wrote", HERE / "sort_known_answers.json", HERE / "step_random_mix_24.npz")


if __name__ == "__main__":
    main()
