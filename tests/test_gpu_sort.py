"""The onesweep radix sort operator (dyn_radix_sort) against numpy's stable sort.

Restates the behaviours crates/dynamis-sort/tests/gpu.rs pins: a stable sort carrying a payload,
two-word keys, and lengths around the tile boundaries.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dynamis_b200 import World
from dynamis_b200._native import check, lib

pytestmark = pytest.mark.gpu


def gpu_sort(world, major, minor, payload, major_digits, minor_digits):
    dev = torch.device("cuda:0")
    tm = torch.from_numpy(major.view(np.int32)).to(dev)
    tn = torch.from_numpy(minor.view(np.int32)).to(dev) if minor is not None else None
    tp = torch.from_numpy(payload.view(np.int32)).to(dev) if payload is not None else None
    torch.cuda.synchronize()
    check(lib.dyn_radix_sort(world._h, tm.data_ptr(), tn.data_ptr() if tn is not None else None,
                             tp.data_ptr() if tp is not None else None, len(major), major_digits, minor_digits), world._h)
    world.wait()
    out = [tm.cpu().numpy().view(np.uint32)]
    out.append(tn.cpu().numpy().view(np.uint32) if tn is not None else None)
    out.append(tp.cpu().numpy().view(np.uint32) if tp is not None else None)
    return out


@pytest.fixture(scope="module")
def world():
    w = World(capacity={"bodies": 1, "colliders": 1, "pairs": 1 << 20})
    from dynamis_b200 import scenes

    scenes.sphere_row(2).build(w)
    w.step(1 / 60)
    w.wait()
    yield w
    w.close()


@pytest.mark.parametrize("n", [1, 7, 255, 256, 257, 1000, 2047, 2048, 2049, 5000, 100000])
def test_stable_with_payload(world, n):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 1 << 12, size=n, dtype=np.uint32)
    payload = np.arange(n, dtype=np.uint32)
    major, _, carried = gpu_sort(world, keys.copy(), None, payload.copy(), 4, 0)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(major, keys[order])
    assert np.array_equal(carried, payload[order])


def test_two_word_keys(world):
    n = 300000
    rng = np.random.default_rng(3)
    major = rng.integers(0, 1 << 18, size=n, dtype=np.uint32)
    minor = rng.integers(0, 1 << 18, size=n, dtype=np.uint32)
    payload = np.arange(n, dtype=np.uint32)
    smaj, smin, spay = gpu_sort(world, major.copy(), minor.copy(), payload.copy(), 3, 3)
    order = np.lexsort((minor, major))
    assert np.array_equal(smaj, major[order])
    assert np.array_equal(smin, minor[order])
    assert np.array_equal(spay, payload[order])


def test_growing_sort_scratch_then_closing_leaves_no_latched_error():
    """Sorting ever larger arrays regrows the world's sort scratch; closing the world afterwards
    must not free anything twice, and the next world's calls must see no stale CUDA error."""
    from dynamis_b200 import scenes

    w = World(capacity={"pairs": 1 << 20})
    scenes.sphere_row(2).build(w)
    w.step(1 / 60)
    w.wait()
    for n in (10, 1000, 100000):
        keys = np.arange(n, 0, -1, dtype=np.uint32)
        out, _, _ = gpu_sort(w, keys.copy(), None, None, 4, 0)
        assert np.array_equal(out, np.sort(keys))
    w.close()
    w2 = World(capacity={"pairs": 1 << 20})
    scenes.sphere_row(2).build(w2)
    w2.step(1 / 60)
    w2.wait()
    keys = np.arange(5000, 0, -1, dtype=np.uint32)
    out, _, _ = gpu_sort(w2, keys.copy(), None, None, 4, 0)
    assert np.array_equal(out, np.sort(keys))
    w2.close()


def test_known_answers_of_the_reference_sort_tests(world):
    """The cases of crates/dynamis-sort/tests/gpu.rs:192-275 from tests/golden/sort_known_answers.json."""
    import hashlib
    import json
    from pathlib import Path

    from test_golden import xorshift_keys

    cases = json.loads((Path(__file__).resolve().parent / "golden" / "sort_known_answers.json").read_text())
    ten = cases["ten_keys"]
    keys = np.array(ten["keys"], np.uint32)
    major, _, payload = gpu_sort(world, keys, None, np.arange(len(keys), dtype=np.uint32), ten["major_digits"], 0)
    assert major.tolist() == ten["sorted"] and payload.tolist() == ten["payload"]
    mm = cases["major_above_minor"]
    major, minor, payload = gpu_sort(world, np.array(mm["major"], np.uint32), np.array(mm["minor"], np.uint32),
                                     np.arange(len(mm["major"]), dtype=np.uint32), mm["major_digits"], mm["minor_digits"])
    assert major.tolist() == mm["sorted_major"] and minor.tolist() == mm["sorted_minor"]
    assert payload.tolist() == mm["payload"]
    wide = cases["wide_two_word"]
    major = xorshift_keys(wide["length"], wide["major_salt"])
    minor = xorshift_keys(wide["length"], wide["minor_salt"])
    smaj, smin, pay = gpu_sort(world, major, minor, np.arange(wide["length"], dtype=np.uint32), wide["major_digits"],
                               wide["minor_digits"])

    def digest(a):
        return hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()

    assert digest(smaj) == wide["sorted_major_sha256"] and digest(smin) == wide["sorted_minor_sha256"]
    assert digest(pay) == wide["payload_sha256"]


def test_a_lookback_wait_that_runs_out_is_reported_and_cleared(world):
    """The bounded look-back wait, made to run out on purpose: the first tile of every digit pass is
    never run (its ticket is skipped), so the later tiles poll for a word nothing writes until their
    limit of 1,000 polls is spent. Every write stays within the n keys. dyn_sync must then report
    DYN_ERR_DEVICE_STATUS with the timeout bit, and after the status is cleared a normal sort and a
    normal step succeed."""
    from dynamis_b200._native import DynamisError

    rng = np.random.default_rng(5)
    n = 5 * 2048 + 17  # six tiles: five of them wait on the missing first one
    keys = rng.integers(0, 1 << 30, size=n, dtype=np.uint32)
    check(lib.dyn_debug_sort_fault(world._h, 1, 1000), world._h)
    tm = torch.from_numpy(keys.view(np.int32)).to("cuda:0")
    torch.cuda.synchronize()
    check(lib.dyn_radix_sort(world._h, tm.data_ptr(), None, None, n, 4, 0), world._h)
    assert lib.dyn_sync(world._h) == 5  # DYN_ERR_DEVICE_STATUS
    status = ctypes.c_uint32(0)
    check(lib.dyn_device_status(world._h, ctypes.byref(status)), world._h)
    assert status.value & 1  # DYN_STATUS_LOOKBACK_TIMEOUT
    with pytest.raises(DynamisError):
        world.wait()
    check(lib.dyn_clear_device_status(world._h), world._h)
    world.wait()
    got = gpu_sort(world, keys, None, None, 4, 0)[0]
    assert np.array_equal(got, np.sort(keys))
    world.step(1 / 60)
    world.wait()
