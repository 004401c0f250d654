"""Build libphaser_b200.so in-tree with nvcc for sm_100a.

    python -m phaser_b200.build                  # or phaser_b200.build.build()
    python -m phaser_b200.build --bounds-check   # also libphaser_b200_bounds.so

The library is a plain C ABI (include/phaser_b200.h); nothing here depends on
torch.  Objects are rebuilt when a source or header is newer than the .so.

The bounds-checking build (-DPHB_BOUNDS_CHECK=1) has the same entry points; its
kernels check every caller-supplied position index against n_pos and report one
outside [0, n_pos) as PHB_STATUS_BOUNDS in the step's status instead of reading or
writing out of bounds.  `phaser_b200._lib` loads it when PHASER_B200_BOUNDS_CHECK=1.
Only the translation units in CHECKED carry checks: the bounds library links their
checked objects with the default build's objects of the others, and its compiles run
beside the default build's.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / 'csrc'
LIB = PKG / 'libphaser_b200.so'
BOUNDS_LIB = PKG / 'libphaser_b200_bounds.so'
SOURCES = ['phb_runtime.cu', 'phb_ops.cu', 'phb_engine.cu', 'phb_optim.cu', 'phb_constraints.cu', 'phb_cnn.cu',
           'phb_prepare.cu']
CHECKED = ['phb_engine.cu']   # the sources whose kernels dereference caller-supplied position indices
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
OBJ_DIR = PKG / '_build'
BOUNDS_OBJ_DIR = PKG / '_build_bounds'


def nvcc() -> str:
    cand = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _stale(lib: Path) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = list(CSRC.glob('*.cu')) + list(CSRC.glob('*.cuh')) + list(CSRC.glob('*.h'))
    deps.append(ROOT / 'include' / 'phaser_b200.h')
    return any(p.stat().st_mtime > t for p in deps)


def _obj(out_dir: Path, src: str) -> Path:
    return out_dir / (Path(src).stem + '.o')


def _compile(sources, out_dir: Path, verbose: bool, defines=()):
    """Start one nvcc per translation unit; returns (source, process) pairs."""
    out_dir.mkdir(exist_ok=True)
    flags = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC',
             '-Xptxas', '-v' if verbose else '-O3', *ARCH, f'-I{ROOT / "include"}', *defines]
    return [(src, subprocess.Popen([nvcc(), '-c', str(CSRC / src), '-o', str(_obj(out_dir, src)), *flags],
                                   stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)) for src in sources]


def _wait(jobs, verbose: bool) -> None:
    for src, proc in jobs:
        _, err = proc.communicate()
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{err}")
        if verbose:
            sys.stderr.write(err)


def _link(lib: Path, objs) -> None:
    tmp = lib.with_suffix('.so.tmp')
    res = subprocess.run([nvcc(), '-shared', '-o', str(tmp), *map(str, objs), *ARCH, '-lcudart'],
                         capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    os.replace(tmp, lib)


def build(force: bool = False, verbose: bool = False, bounds_check: bool = False) -> Path:
    """Build libphaser_b200.so when it is stale (or `force`); with `bounds_check` also
    libphaser_b200_bounds.so, compiled at the same time.  Returns the library asked for."""
    main = force or _stale(LIB) or not all(_obj(OBJ_DIR, s).exists() for s in SOURCES)
    bounds = bounds_check and (main or _stale(BOUNDS_LIB))
    jobs = _compile(SOURCES, OBJ_DIR, verbose) if main else []
    checked = _compile(CHECKED, BOUNDS_OBJ_DIR, verbose, ['-DPHB_BOUNDS_CHECK=1']) if bounds else []
    _wait(jobs, verbose)   # the translation units of both libraries compile in parallel
    if main:
        _link(LIB, [_obj(OBJ_DIR, s) for s in SOURCES])
    if bounds:
        _wait(checked, verbose)
        _link(BOUNDS_LIB, [_obj(BOUNDS_OBJ_DIR if s in CHECKED else OBJ_DIR, s) for s in SOURCES])
    return BOUNDS_LIB if bounds_check else LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv, bounds_check='--bounds-check' in sys.argv))
