"""The C-ABI library loads without a GPU and exports every symbol include/ffxcuda.h declares."""
import ctypes
import os
import re

from forcefieldx_b200 import cabi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "ffxcuda.h")).read()
    return sorted(set(re.findall(r"\b(ffxg_[A-Za-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(cabi.PROTOTYPES)


def test_library_exports_every_declared_symbol():
    lib = cabi.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_struct_sizes_match_header_layout():
    # Offsets of a few fields pin the ctypes mirror to the C layout.
    assert cabi.FfxgParams.box.offset == 0
    assert cabi.FfxgParams.pme_grid.offset == 8 * 3 + 8 * 5
    assert cabi.FfxgSystem.xyz.offset == 8


def test_create_rejects_bad_arguments_without_touching_a_device():
    lib = cabi.load_library()
    h = ctypes.c_void_p()
    st = lib.ffxg_create(None, None, ctypes.byref(h))
    assert st == 1  # FFXG_ERR_BAD_ARG
