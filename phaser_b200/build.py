"""Build libphaser_b200.so in-tree with nvcc for sm_100a.

    python -m phaser_b200.build                  # or phaser_b200.build.build()
    python -m phaser_b200.build --bounds-check   # libphaser_b200_bounds.so

The library is a plain C ABI (include/phaser_b200.h); nothing here depends on
torch.  Objects are rebuilt when a source or header is newer than the .so.

The bounds-checking build (-DPHB_BOUNDS_CHECK=1) has the same entry points; its
kernels check every caller-supplied position index against n_pos and report one
outside [0, n_pos) as PHB_STATUS_BOUNDS in the step's status instead of reading or
writing out of bounds.  `phaser_b200._lib` loads it when PHASER_B200_BOUNDS_CHECK=1.
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
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


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


def build(force: bool = False, verbose: bool = False, bounds_check: bool = False) -> Path:
    lib = BOUNDS_LIB if bounds_check else LIB
    if not force and not _stale(lib):
        return lib
    out_dir = PKG / ('_build_bounds' if bounds_check else '_build')
    out_dir.mkdir(exist_ok=True)
    flags = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC',
             '-Xptxas', '-v' if verbose else '-O3', *ARCH, f'-I{ROOT / "include"}']
    if bounds_check:
        flags.append('-DPHB_BOUNDS_CHECK=1')
    objs = [str(out_dir / (Path(src).stem + '.o')) for src in SOURCES]
    procs = [subprocess.Popen([nvcc(), '-c', str(CSRC / src), '-o', obj, *flags], stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, text=True) for src, obj in zip(SOURCES, objs)]
    for src, proc in zip(SOURCES, procs):   # the translation units compile in parallel
        _, err = proc.communicate()
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{err}")
        if verbose:
            sys.stderr.write(err)
    tmp = lib.with_suffix('.so.tmp')
    cmd = [nvcc(), '-shared', '-o', str(tmp), *objs, *ARCH, '-lcudart']
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    os.replace(tmp, lib)
    return lib


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv, bounds_check='--bounds-check' in sys.argv))
