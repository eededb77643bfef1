"""The C ABI library loads and exports every entry point include/*.h declares
(no device calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

from canoe_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    inc = os.path.join(ROOT, "include")
    for f in sorted(os.listdir(inc)):
        if not f.endswith(".h"):
            continue
        src = open(os.path.join(inc, f)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(canoe_[a-z_0-9]+)\s*\(", src, re.M)
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    assert "canoe_block_step" in names and "canoe_riemann_hllc" in names
    assert len(names) == len(set(names))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    bound = {n for n, _, _ in _abi.SIGNATURES}
    declared = set(declared_functions())
    assert declared - bound == set(), sorted(declared - bound)
    assert bound - declared == set(), sorted(bound - declared)


def test_struct_layouts_match_header():
    # sizes computed from the C declarations (natural alignment, x86-64)
    assert ctypes.sizeof(_abi.Thermo) == 8 + 3 * 8 + 3 * 8 * 8 + 2 * 4 * 4 + 6 * 8 * 4
    assert ctypes.sizeof(_abi.SatOpts) == 16
    assert _abi.BlockConfig.thermo.offset % 8 == 0


def test_version_string():
    assert b"sm_100a" in _abi.load().canoe_version()
