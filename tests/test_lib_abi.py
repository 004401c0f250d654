"""The C-ABI library loads and exports every entry point the header declares
(CPU only: no call touches a GPU)."""
import ctypes
import os
import re

from phaser_b200 import _lib

from .conftest import ROOT


def header_functions():
    text = open(os.path.join(ROOT, 'include', 'phaser_b200.h')).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(phb_[a-z0-9_]+)\s*\(', text)))


def test_library_loads_and_exports_header_symbols():
    lib = _lib.load()
    declared = header_functions()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in the header but not exported"
    # the Python binding covers every declared entry point
    assert set(declared) <= set(_lib.EXPORTED), set(declared) - set(_lib.EXPORTED)


def test_host_only_entry_points():
    lib = _lib.load()
    assert lib.phb_version() >= 100
    assert lib.phb_status_string(_lib.PHB_OK) == b'ok'
    assert lib.phb_status_string(_lib.PHB_ERR_UNSUPPORTED).startswith(b'unsupported')
    # workspace sizing is host arithmetic
    n = lib.phb_engine_workspace_bytes(128, 4, 8, 256, 517, 517)
    psi = 256 * 4 * 8 * 128 * 128 * 8
    assert psi < n < psi + 64 * 2 ** 20
    assert lib.phb_engine_workspace_bytes(0, 4, 8, 256, 517, 517) == 0


def test_struct_layouts_match_header():
    # phb_engine: 4 int32, 3 int64, 4 double, 10 pointers, int32 + 3 float, pointer, size_t, 2 pointers
    p = ctypes.sizeof(ctypes.c_void_p)
    assert ctypes.sizeof(_lib.PhbEngine) == 16 + 24 + 32 + 10 * p + 16 + p + 8 + 2 * p
    assert _lib.PhbStep.pos_update.offset == 32


def test_invalid_arguments_are_rejected_without_a_gpu():
    lib = _lib.load()
    # null pointers are rejected before any CUDA call
    assert lib.phb_fft2_c64(None, None, 1, 128, 0, None) == _lib.PHB_ERR_INVALID_ARG
    assert lib.phb_cutout_get_c64(None, 1, 1, 1, None, 1, 1, 1, 1.0, 0.0, None, None) == _lib.PHB_ERR_INVALID_ARG
    assert lib.phb_solver_group(None, None, None, 0, None) == _lib.PHB_ERR_INVALID_ARG
