"""The C-ABI library builds, loads without a GPU and exports every entry point
include/ibisco_gpu.h declares (no compute call is made here)."""
import ctypes
import os
import re

from ibisco_b200 import build, native

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "ibisco_gpu.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ibg_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_abi():
    names = declared()
    for n in ("ibg_create", "ibg_set_state", "ibg_step", "ibg_run", "ibg_get_state", "ibg_get_neighbour_list",
              "ibg_get_exclusions", "ibg_last_error", "ibg_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(native.EXPORTS) <= set(declared())


def test_version_string_without_gpu():
    assert b"sm_100a" in native.lib().ibg_version()


def test_create_rejects_null_descriptor():
    h = ctypes.c_void_p()
    assert native.lib().ibg_create(None, 0, ctypes.byref(h)) == -1
