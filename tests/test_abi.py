"""The boundary's data contract: record layouts, exported symbols, the header compiles.

Offsets restate what crates/dynamis-abi/tests/records.rs:241-276 and 1065-1071 pin for the WGSL
storage layouts (records.wgsl); the C header asserts the same offsets at compile time.
"""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from dynamis_b200 import records as R

ROOT = Path(__file__).resolve().parent.parent


def test_collider_layout():
    d = R.COLLIDER
    assert d.itemsize == 112
    assert d.fields["relaxation"][1] == 20
    assert d.fields["damping_ratio"][1] == 24
    assert d.fields["half_extents"][1] == 32


def test_contact_layout():
    d = R.CONTACT
    assert d.itemsize == 352
    expect = {"events": 44, "surface": 48, "triangle": 52, "friction": 56, "carried_normal": 72,
              "carried_tangent": 76, "relaxation": 80, "damping_ratio": 84, "points": 96}
    for name, offset in expect.items():
        assert d.fields[name][1] == offset, name
    mp = R.MANIFOLD_POINT
    assert mp.itemsize == 64
    assert mp.fields["accumulated_normal"][1] == 44
    assert mp.fields["accumulated_tangent_1"][1] == 48
    assert mp.fields["accumulated_tangent_2"][1] == 52
    assert mp.fields["feature"][1] == 56


def test_body_layouts():
    assert R.BODY_STATE.itemsize == 144
    assert R.BODY_STATE.fields["velocity"][1] == 64
    assert R.BODY_STATE.fields["body_id"][1] == 128
    assert R.BODY_DESCRIPTOR.itemsize == 128
    assert R.BODY_DESCRIPTOR.fields["com"][1] == 48
    assert R.BODY_DESCRIPTOR.fields["inverse_inertia"][1] == 88
    assert R.STEP_PARAMS.itemsize == 176


@pytest.mark.parametrize("compiler,flag", [("gcc", "-std=c11"), ("g++", "-std=c++17")])
def test_headers_compile_with_static_layout_asserts(tmp_path, compiler, flag):
    src = tmp_path / ("t.c" if compiler == "gcc" else "t.cpp")
    src.write_text('#include "dynamis_cuda.h"\nint main(void) { return (int)sizeof(dyn_contact_record) - 352; }\n')
    proc = subprocess.run([compiler, flag, "-I", str(ROOT / "include"), str(src), "-o", str(tmp_path / "t")],
                          capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr
    assert subprocess.run([str(tmp_path / "t")]).returncode == 0


def test_descriptor_structs_match_numpy(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include "dynamis_cuda.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu\\n", sizeof(dyn_config), sizeof(dyn_capacity),'
                   ' sizeof(dyn_collider_desc), sizeof(dyn_body_desc)); return 0; }\n')
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(tmp_path / "s")], check=True)
    out = subprocess.run([str(tmp_path / "s")], capture_output=True, text=True).stdout.split()
    assert [int(x) for x in out] == [R.CONFIG.itemsize, R.CAPACITY.itemsize, R.COLLIDER_DESC.itemsize,
                                     R.BODY_DESC.itemsize]


def declared_symbols():
    text = (ROOT / "include" / "dynamis_cuda.h").read_text()
    return sorted(set(re.findall(r"DYN_API\s+[\w\s\*]+?\b(dyn_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from dynamis_b200 import _native

    lib_path = _native.LIBRARY
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (dyn_\w+)", out))
    declared = declared_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    unbound = [s for s in declared if s not in _native.SIGNATURES]
    assert not unbound, f"declared but not bound in _native: {unbound}"


def test_abi_version_and_status_strings():
    from dynamis_b200 import lib

    assert lib.dyn_abi_version() == 1
    assert lib.dyn_status_string(0) == b"ok"
    assert b"capacity" in lib.dyn_status_string(2)


def test_counter_slots_follow_the_reference_declaration_order():
    # crates/dynamis-abi/src/counter.rs:76-128
    assert R.COUNTER["ENTRIES"] == 0
    assert R.COUNTER["PAIRS"] == 10
    assert R.COUNTER["CONTACTS"] == 12
    assert R.COUNTER["ISLANDS"] == 28
    assert R.COUNTER["GRID_SCALE"] == 35
    assert R.COUNTER["LIVE"] == 40
    assert R.COUNTER["REFUSED_SOFT_EVENTS"] == 51
    assert len(R.COUNTERS) == R.COUNTER_DEVICE_COUNT == 52


def test_the_rust_binding_declares_every_entry_point():
    """integration/dynamis-cuda-sys/src/lib.rs (the crate a Dynamis maintainer adds; no Rust toolchain
    here) declares exactly the entry points include/dynamis_cuda.h exports."""
    import re
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    header = re.sub(r"/\*.*?\*/", "", (root / "include" / "dynamis_cuda.h").read_text(), flags=re.S)
    exported = set(re.findall(r"DYN_API\s+[^;(]*?\b(dyn_\w+)\s*\(", header))
    rust = set(re.findall(r"pub fn (dyn_\w+)\(", (root / "integration" / "dynamis-cuda-sys" / "src" / "lib.rs").read_text()))
    assert exported and rust == exported, (exported - rust, rust - exported)
