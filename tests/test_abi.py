"""CPU checks of the C-ABI library: it loads without a GPU and exports every
function that include/*.h declares; no compute calls here."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w ]+?\**\s*\b(ispan\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from ispan_b200 import _lib
    L = _lib.lib()
    names = declared("ispan_b200.h")
    assert "ispan_scc_run" in names and "ispan_ctx_create" in names
    for n in names:
        assert hasattr(L, n), n
    assert set(_lib.SYMBOLS) <= set(names)


def test_gen_library_exports():
    path = os.path.join(ROOT, "ispan_b200", "libispan_gen.so")
    if not os.path.exists(os.path.join(ROOT, "include", "ispan_gen.h")):
        pytest.skip("no generator header")
    L = ctypes.CDLL(path)
    for n in declared("ispan_gen.h"):
        assert hasattr(L, n), n


def test_version_and_errors_without_gpu():
    from ispan_b200 import _lib
    L = _lib.lib()
    assert b"sm_100a" in L.ispan_version()
    assert L.ispan_strerror(-4) == b"device-side wait timed out"
    h = ctypes.c_void_p()
    import torch
    if not torch.cuda.is_available():
        assert L.ispan_ctx_create(0, 10, 10, ctypes.byref(h)) == -6  # ISPAN_ERR_NODEV, no crash


def test_flag_values_match_the_header():
    """The Python binding's run flags carry the header's values."""
    from ispan_b200 import _lib
    src = open(os.path.join(ROOT, "include", "ispan_b200.h")).read()
    flags = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define ISPAN_F_(\w+)\s+(\d+)u", src)}
    assert {"LABELS_ON_DEVICE", "VALIDATE", "EXACT_STATS", "REVERSE_ATOMIC"} <= set(flags)
    for name, value in flags.items():
        if hasattr(_lib, "F_" + name):
            assert getattr(_lib, "F_" + name) == value, name
    assert _lib.F_REVERSE_ATOMIC == flags["REVERSE_ATOMIC"]
