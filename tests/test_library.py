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


def header_defines(prefix):
    src = open(HEADER).read()
    return {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(" + prefix + r"[A-Z0-9_]*)\s+\(?(-?\d+)\)?", src)}


def test_constants_match_the_header():
    """The binding's precision, centre-of-mass and list-form constants are the
    header's."""
    d = header_defines("IBG_")
    assert d["IBG_PREC_FP32_FIXED"] == native.IBG_PREC_FP32_FIXED
    assert d["IBG_PREC_FP64_PLAIN"] == native.IBG_PREC_FP64_PLAIN
    assert d["IBG_VS_COM_FIXED"] == native.IBG_VS_COM_FIXED
    assert d["IBG_VS_COM_REFERENCE"] == native.IBG_VS_COM_REFERENCE
    assert d["IBG_LIST_AUTO"] == native.LIST_AUTO
    assert d["IBG_LIST_PER_PARTICLE"] == native.LIST_PER_PARTICLE
    assert d["IBG_LIST_PER_SLICE"] == native.LIST_PER_SLICE


def test_list_form_rejects_bad_arguments_without_gpu():
    assert native.lib().ibg_set_list_form(None, native.LIST_PER_SLICE) == -1
    assert native.lib().ibg_get_list_form(None) == -1


def test_fortran_parameters_match_the_header():
    """The Fortran module's named constants are the header's."""
    src = open(os.path.join(os.path.dirname(HEADER), "..", "fortran", "ibisco_gpu_mod.f90")).read()
    params = {m.group(1): int(m.group(2)) for m in re.finditer(r"\b(IBG_[A-Z0-9_]+)\s*=\s*(-?\d+)", src)}
    d = header_defines("IBG_")
    assert params, "no PARAMETER constants found"
    for name, value in params.items():
        assert d[name] == value, name
