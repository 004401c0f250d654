"""The C-ABI library loads and exports every entry point the header declares
(CPU only: no call touches a GPU)."""
import ctypes
import os
import re
import subprocess
import sys

import pytest

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


def test_header_constants_match_the_binding():
    text = open(os.path.join(ROOT, 'include', 'phaser_b200.h')).read()
    found = 0
    for name, val in re.findall(r'^#define (PHB_[A-Z0-9_]+)\s+(\d+|\(1 << \d+\))', text, flags=re.M):
        want = 1 << int(val[6:-1]) if val.startswith('(') else int(val)
        if hasattr(_lib, name):
            assert getattr(_lib, name) == want, name
            found += 1
    assert found >= 18


def test_bounds_checking_build_exports_the_same_entry_points():
    """libphaser_b200_bounds.so (build(bounds_check=True): kernels compiled with
    -DPHB_BOUNDS_CHECK=1) has every entry point of the header, and the loader picks
    it when PHASER_B200_BOUNDS_CHECK=1."""
    from phaser_b200 import build as B
    path = B.build(bounds_check=True)   # nothing to do when it is newer than the sources
    lib = ctypes.CDLL(str(path))
    for name in header_functions():
        assert hasattr(lib, name), f"{name} missing from the bounds-checking build"
    code = "import os; from phaser_b200 import _lib; print(os.path.basename(_lib.load()._name))"
    for flag, want in (('1', 'libphaser_b200_bounds.so'), ('0', 'libphaser_b200.so')):
        env = dict(os.environ, PHASER_B200_BOUNDS_CHECK=flag)
        got = subprocess.run([sys.executable, '-c', code], cwd=ROOT, env=env, capture_output=True, text=True,
                             check=True).stdout.strip()
        assert got == want


def test_step_status_words_map_to_exceptions():
    _lib.raise_for_status(-1)
    with pytest.raises(ValueError, match='group 3'):
        _lib.raise_for_status(3)
    with pytest.raises(IndexError, match='group 4'):
        _lib.raise_for_status(_lib.PHB_STATUS_BOUNDS | 4)
    with pytest.raises(RuntimeError, match='group 5'):
        _lib.raise_for_status(_lib.PHB_STATUS_INTERNAL | 5)


def test_host_only_entry_points():
    lib = _lib.load()
    assert lib.phb_version() >= 100
    assert lib.phb_status_string(_lib.PHB_OK) == b'ok'
    assert lib.phb_status_string(_lib.PHB_ERR_UNSUPPORTED).startswith(b'unsupported')
    # workspace sizing is host arithmetic
    n = lib.phb_engine_workspace_bytes(128, 4, 8, 256, 517, 517)
    psi = 256 * 4 * 8 * 128 * 128 * 8                     # per-slice incident waves
    far = 256 * 4 * 128 * 128 * 8 + 256 * 128 * 128 * 4   # far-field waves and intensities
    assert psi + far < n < psi + far + 64 * 2 ** 20
    assert lib.phb_engine_workspace_bytes(0, 4, 8, 256, 517, 517) == 0


STRUCTS = {'phb_engine': _lib.PhbEngine, 'phb_step': _lib.PhbStep, 'phb_optim': _lib.PhbOptim,
           'phb_obj_reg': _lib.PhbObjReg, 'phb_probe_reg': _lib.PhbProbeReg}


def test_struct_layouts_match_header(tmp_path):
    """Every field offset and struct size of the ctypes mirrors against the C
    compiler's view of include/phaser_b200.h (gcc on a generated probe)."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "phaser_b200.h"', 'int main(void) {']
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ['return 0;', '}']
    src = tmp_path / 'probe.c'
    src.write_text('\n'.join(lines))
    exe = tmp_path / 'probe'
    subprocess.run(['gcc', '-std=c11', '-I', os.path.join(ROOT, 'include'), str(src), '-o', str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split('\n')
    seen = 0
    for line in filter(None, out):
        cname, field, val = line.split()
        py = STRUCTS[cname]
        want = ctypes.sizeof(py) if field == 'size' else getattr(py, field).offset
        assert int(val) == want, (cname, field)
        seen += 1
    assert seen == sum(len(py._fields_) + 1 for py in STRUCTS.values())


def test_invalid_arguments_are_rejected_without_a_gpu():
    lib = _lib.load()
    # null pointers are rejected before any CUDA call
    assert lib.phb_fft2_c64(None, None, 1, 128, 0, None) == _lib.PHB_ERR_INVALID_ARG
    assert lib.phb_cutout_get_c64(None, 1, 1, 1, None, 1, 1, 1, 1.0, 0.0, None, None) == _lib.PHB_ERR_INVALID_ARG
    assert lib.phb_solver_group(None, None, None, 0, None) == _lib.PHB_ERR_INVALID_ARG
    # the allocation-free step refuses a partial (data-parallel) launch before any CUDA call
    desc, st = _lib.PhbEngine(), _lib.PhbStep()
    st.flags = _lib.PHB_FLAG_PARTIAL
    grp = (ctypes.c_int64 * 1)(0)
    assert lib.phb_solver_group_static(ctypes.byref(desc), ctypes.byref(st), grp, 1, None) == _lib.PHB_ERR_UNSUPPORTED
    # the wait probe takes 1 .. 2^22 attempts (the limit of the tensor-core kernels' waits)
    out = (ctypes.c_int32 * 1)(0)
    assert lib.phb_wait_probe(0, 16, None, None) == _lib.PHB_ERR_INVALID_ARG
    assert lib.phb_wait_probe(0, 0, out, None) == _lib.PHB_ERR_INVALID_ARG
    assert lib.phb_wait_probe(0, (1 << 22) + 1, out, None) == _lib.PHB_ERR_INVALID_ARG
    assert lib.phb_wait_probe(2, 16, out, None) == _lib.PHB_ERR_INVALID_ARG


def test_argument_checks_return_status_without_touching_a_gpu():
    """Entry points reject null pointers and impossible sizes with a status code, before
    any CUDA call (so this runs without a GPU).  Pointer arguments here are never
    dereferenced: every call fails its argument check first."""
    lib = _lib.load()
    bad = _lib.PHB_ERR_INVALID_ARG
    fake = ctypes.c_void_p(0x1000)   # non-null but never used: the size checks fail first
    # resampling: null input, empty shapes
    assert lib.phb_resample_c64(None, 1, 8, 8, fake, 8, 8, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0, None) == bad
    assert lib.phb_resample_f32(fake, 0, 8, 8, fake, 8, 8, 1.0, 1.0, 0.0, 0.0, 0.0, 0, None) == bad
    assert lib.phb_resample_f32(fake, 1, 8, 8, fake, 0, 8, 1.0, 1.0, 0.0, 0.0, 0.0, 0, None) == bad
    # reslicing: too many slices, bad padding mode, null tables
    i32 = (ctypes.c_int32 * 1)(1)
    f32 = (ctypes.c_float * 1)(1.0)
    assert lib.phb_resample_slices_c64(fake, 200, 16, f32, fake, 1, f32, i32, i32, f32, f32, 0, None) == bad
    assert lib.phb_resample_slices_c64(fake, 1, 16, f32, fake, 1, f32, i32, i32, f32, f32, 3, None) == bad
    assert lib.phb_resample_slices_c64(fake, 1, 16, None, fake, 1, f32, i32, i32, f32, f32, 0, None) == bad
    # warm-start helpers: windows that do not divide, empty batches
    assert lib.phb_pattern_features(fake, None, 1, 64, 63, 1, 0, fake, None) == bad
    assert lib.phb_pattern_features(fake, None, 1, 64, 128, 1, 0, fake, None) == bad
    assert lib.phb_pattern_features(fake, None, 0, 64, 64, 1, 0, fake, None) == bad
    assert lib.phb_stitch_patches(None, fake, None, 1, 0.0, 0.0, 1.0, 1.0, 64, 32, None, fake, fake, 8, 8, None) == bad
    assert lib.phb_stitch_patches(fake, fake, None, 1, 0.0, 0.0, 1.0, 1.0, 64, 65, None, fake, fake, 8, 8, None) == bad
    assert lib.phb_conv3x3_fwd(None, fake, fake, fake, 1, 1, 8, 8, 1, 1, 0, None) == bad
    assert lib.phb_conv3x3_fwd(fake, fake, fake, fake, 1, 1, 8, 8, 1, 3, 0, None) == _lib.PHB_ERR_UNSUPPORTED
