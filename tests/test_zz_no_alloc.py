"""dyn_radix_sort_static: the sort entry point that allocates nothing, against dyn_radix_sort.

Some callers cannot allocate device memory: they own it all through their own pool, or they run
on a path where cudaMalloc / cudaFree would synchronise the device. For them the library keeps the
sort's scratch in a fixed device array of its own. This file checks, on the GPU and through the
C ABI, that two calls in a row (with different sizes and key shapes, so a previous call's leftovers
in the shared array would show) give exactly what the allocating entry point gives, and that a
request above the array's capacity is refused. It runs alone or after every other test.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dynamis_b200 import World, scenes
from dynamis_b200._native import check, lib

pytestmark = pytest.mark.gpu

MAX_KEYS = 262144  # DYN_STATIC_SORT_MAX_KEYS


def device_copy(array):
    return None if array is None else torch.from_numpy(array.view(np.int32)).to("cuda:0")


def host(t):
    return None if t is None else t.cpu().numpy().view(np.uint32)


def sort_with_world(world, major, minor, payload, major_digits, minor_digits):
    tm, tn, tp = device_copy(major), device_copy(minor), device_copy(payload)
    torch.cuda.synchronize()
    check(lib.dyn_radix_sort(world._h, tm.data_ptr(), tn.data_ptr() if tn is not None else None,
                             tp.data_ptr() if tp is not None else None, len(major), major_digits, minor_digits), world._h)
    world.wait()
    return host(tm), host(tn), host(tp)


def sort_static(major, minor, payload, major_digits, minor_digits):
    tm, tn, tp = device_copy(major), device_copy(minor), device_copy(payload)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    status = lib.dyn_radix_sort_static(tm.data_ptr(), tn.data_ptr() if tn is not None else None,
                                       tp.data_ptr() if tp is not None else None, len(major), major_digits,
                                       minor_digits, stream.cuda_stream)
    assert status == 0, f"dyn_radix_sort_static returned {status}"
    torch.cuda.synchronize()
    return host(tm), host(tn), host(tp)


@pytest.fixture(scope="module")
def world():
    w = World(capacity={"pairs": 1 << 20})
    scenes.sphere_row(2).build(w)
    w.step(1 / 60)
    w.wait()
    yield w
    w.close()


def test_two_calls_in_a_row_match_the_allocating_sort(world):
    rng = np.random.default_rng(11)
    # call 1: two-word keys with a payload, at the capacity limit
    n1 = MAX_KEYS
    major = rng.integers(0, 1 << 18, size=n1, dtype=np.uint32)
    minor = rng.integers(0, 1 << 18, size=n1, dtype=np.uint32)
    payload = np.arange(n1, dtype=np.uint32)
    want = sort_with_world(world, major, minor, payload, 3, 3)
    got = sort_static(major, minor, payload, 3, 3)
    for w_, g_ in zip(want, got):
        assert np.array_equal(w_, g_)
    order = np.lexsort((minor, major))
    assert np.array_equal(got[0], major[order]) and np.array_equal(got[2], payload[order])
    # call 2: fewer one-word keys over an odd number of digit passes
    n2 = 70001
    keys = rng.integers(0, 1 << 24, size=n2, dtype=np.uint32)
    payload2 = rng.integers(0, 1 << 32, size=n2, dtype=np.uint64).astype(np.uint32)
    want = sort_with_world(world, keys, None, payload2, 3, 0)
    got = sort_static(keys, None, payload2, 3, 0)
    assert np.array_equal(want[0], got[0]) and np.array_equal(want[2], got[2])
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(got[0], keys[order]) and np.array_equal(got[2], payload2[order])


def test_requests_above_the_capacity_are_refused():
    keys = torch.zeros(MAX_KEYS + 1, dtype=torch.int32, device="cuda:0")
    status = lib.dyn_radix_sort_static(keys.data_ptr(), None, None, MAX_KEYS + 1, 4, 0, None)
    assert status == 2  # DYN_ERR_CAPACITY


@pytest.mark.parametrize("with_minor,with_payload,major_digits,minor_digits", [
    (True, False, 2, 2),    # two words, no payload
    (False, False, 3, 0),   # one word, no payload, odd pass count
    (True, True, 0, 3),     # minor digits only (the major word rides along), odd pass count
    (True, False, 0, 2),    # minor digits only, no payload
])
def test_every_kernel_variant_matches_the_allocating_sort(world, with_minor, with_payload, major_digits, minor_digits):
    rng = np.random.default_rng(17 + 4 * major_digits + minor_digits)
    n = 40961
    major = rng.integers(0, 1 << 24, size=n, dtype=np.uint32)
    minor = rng.integers(0, 1 << 24, size=n, dtype=np.uint32) if with_minor else None
    payload = np.arange(n, dtype=np.uint32)[::-1].copy() if with_payload else None
    want = sort_with_world(world, major, minor, payload, major_digits, minor_digits)
    got = sort_static(major, minor, payload, major_digits, minor_digits)
    for w_, g_ in zip(want, got):
        assert (w_ is None and g_ is None) or np.array_equal(w_, g_)
    mask_major = (1 << (8 * major_digits)) - 1
    mask_minor = (1 << (8 * minor_digits)) - 1
    keys = [minor & mask_minor] if with_minor else []
    order = np.lexsort(keys + [major & mask_major])  # stable on the sorted digits only
    assert np.array_equal(got[0], major[order])
    if with_minor:
        assert np.array_equal(got[1], minor[order])
    if with_payload:
        assert np.array_equal(got[2], payload[order])


def test_the_status_of_a_call_is_readable_after_it():
    """A look-back wait made to run out (the first tile's ticket skipped, 1,000 polls) is reported by
    dyn_radix_sort_static_status; the next call clears it."""
    import ctypes

    rng = np.random.default_rng(23)
    n = 4 * 2048 + 5
    keys = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    stream = torch.cuda.current_stream()
    status = ctypes.c_uint32(7)
    sort_static(keys, None, None, 4, 0)
    assert lib.dyn_radix_sort_static_status(stream.cuda_stream, ctypes.byref(status)) == 0 and status.value == 0
    assert lib.dyn_debug_sort_fault(None, 1, 1000) == 0
    sort_static(keys, None, None, 4, 0)
    assert lib.dyn_radix_sort_static_status(stream.cuda_stream, ctypes.byref(status)) == 5  # DYN_ERR_DEVICE_STATUS
    assert status.value & 1  # DYN_STATUS_LOOKBACK_TIMEOUT
    got = sort_static(keys, None, None, 4, 0)[0]
    assert lib.dyn_radix_sort_static_status(stream.cuda_stream, ctypes.byref(status)) == 0 and status.value == 0
    assert np.array_equal(got, np.sort(keys))
