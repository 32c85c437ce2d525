"""The C-ABI library builds for sm_100a, loads, and exports every entry point
that include/elegant_b200.h declares (no GPU work is done here)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "elegant_b200", "libelegant_b200.so")
HEADER = os.path.join(ROOT, "include", "elegant_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^[A-Za-z_][\w \*]*?\b(b2e_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build the engine first (python -m elegant_b200.build)"
    lib = ctypes.CDLL(LIB)
    names = declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (b2e_\w+)", out))
    assert set(names) <= exported


def test_build_targets_sm100a():
    from elegant_b200 import build
    assert "arch=compute_100a,code=sm_100a" in build.NVCC_FLAGS
    assert "--fmad=false" in build.NVCC_FLAGS


def test_version_and_null_handling():
    lib = ctypes.CDLL(LIB)
    assert lib.b2e_version() >= 1
    lib.b2e_last_error.restype = ctypes.c_char_p
    assert lib.b2e_last_error(None) == b"null context"
    assert lib.b2e_destroy(None) == -1


def test_element_defaults_match_the_host_tables():
    """b2e_element_defaults (no device needed) gives every supported type the
    same defaults the Python layer writes, the reference's parameter-table
    values; the CSR filter cutoffs default to -1 (off)."""
    from elegant_b200 import _native as nat
    from elegant_b200.lattice import DEFAULTS, SLOTS, TYPE_NAMES
    lib = ctypes.CDLL(LIB)
    for code in TYPE_NAMES:
        el = nat.Element()
        assert lib.b2e_element_defaults(code, ctypes.byref(el)) == 0
        assert el.type == code
        want = [0.0] * nat.MAX_PARAMS
        for k, v in DEFAULTS.get(code, {}).items():
            want[SLOTS[code][k]] = float(v)
        assert list(el.p) == want, TYPE_NAMES[code]
    el = nat.Element()
    lib.b2e_element_defaults(nat.CSRCSBEND, ctypes.byref(el))
    assert [el.p[i] for i in (31, 32, 33, 34)] == [-1.0] * 4
    assert lib.b2e_element_defaults(99, ctypes.byref(el)) == -1
    assert lib.b2e_element_defaults(nat.DRIF, None) == -1
