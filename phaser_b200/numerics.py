"""Array-level numerics on device tensors through the C ABI.

The B200 counterparts of phaser/utils/num.py (fft2 / ifft2) and
phaser/utils/object.py (ObjectCutout get / add / set).  Tensors are torch CUDA
tensors (torch only provides the device memory and the stream); every
operation runs a libphaser_b200 kernel on the current stream.
"""
from __future__ import annotations

import typing as t

import numpy
import torch

from . import _lib
from .sampling import ObjectSampling


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _check(t_: torch.Tensor, dtype: torch.dtype, name: str) -> None:
    if not t_.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (the B200 backend has no CPU path)")
    if t_.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t_.dtype}")
    if not t_.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def fft2(a: torch.Tensor) -> torch.Tensor:
    """phaser fft2: centred real space, orthonormal (phaser/utils/num.py:460-468)."""
    _check(a, torch.complex64, 'a')
    n = a.shape[-1]
    if a.shape[-2] != n:
        raise ValueError("fft2 needs square N x N tiles")
    out = torch.empty_like(a)
    _lib.call('phb_fft2_c64', a.data_ptr(), out.data_ptr(), a.numel() // (n * n), n, 0, _stream())
    return out


def ifft2(a: torch.Tensor) -> torch.Tensor:
    """phaser ifft2 (phaser/utils/num.py:434-442)."""
    _check(a, torch.complex64, 'a')
    n = a.shape[-1]
    if a.shape[-2] != n:
        raise ValueError("ifft2 needs square N x N tiles")
    out = torch.empty_like(a)
    _lib.call('phb_fft2_c64', a.data_ptr(), out.data_ptr(), a.numel() // (n * n), n, 1, _stream())
    return out


def cutout_starts(sampling: ObjectSampling, scan: torch.Tensor, cutout_shape: t.Tuple[int, int],
                  group: t.Optional[torch.Tensor] = None, with_subpx: bool = False):
    """Integer starts (B, 2) int64 (and sub-pixel shifts (B, 2) float32) of cutouts
    around scan positions, computed on the device bit-exactly as
    phaser/utils/object.py:291-331."""
    _check(scan, torch.float32, 'scan')
    B = scan.numel() // 2 if group is None else group.numel()
    starts = torch.empty((B, 2), dtype=torch.int64, device=scan.device)
    subpx = torch.empty((B, 2), dtype=torch.float32, device=scan.device) if with_subpx else None
    _lib.call('phb_cutout_starts', scan.data_ptr(), 0 if group is None else group.data_ptr(), B,
              float(sampling.corner[0]), float(sampling.corner[1]), float(sampling.sampling[0]),
              float(sampling.sampling[1]), int(cutout_shape[0]), int(cutout_shape[1]),
              starts.data_ptr(), 0 if subpx is None else subpx.data_ptr(), _stream())
    return (starts, subpx) if with_subpx else starts


def _obj_dims(obj: torch.Tensor) -> t.Tuple[int, int, int]:
    S = int(numpy.prod(obj.shape[:-2])) if obj.dim() > 2 else 1
    return S, obj.shape[-2], obj.shape[-1]


def get_cutouts(obj: torch.Tensor, starts: torch.Tensor, shape: t.Tuple[int, int], fill=1.0) -> torch.Tensor:
    """(B, *obj.shape[:-2], ny, nx) cutouts; out-of-bounds reads `fill`
    (ObjectCutout.get, phaser/utils/object.py:501-519)."""
    S, H, W = _obj_dims(obj)
    B = starts.shape[0]
    out = torch.empty((B, *obj.shape[:-2], *shape), dtype=obj.dtype, device=obj.device)
    if obj.dtype == torch.complex64:
        fill = complex(fill)
        _lib.call('phb_cutout_get_c64', obj.data_ptr(), S, H, W, starts.data_ptr(), B, shape[0], shape[1],
                  fill.real, fill.imag, out.data_ptr(), _stream())
    elif obj.dtype == torch.float32:
        _lib.call('phb_cutout_get_f32', obj.data_ptr(), S, H, W, starts.data_ptr(), B, shape[0], shape[1],
                  float(fill), out.data_ptr(), _stream())
    else:
        raise TypeError(f"unsupported dtype {obj.dtype}")
    return out


def add_cutouts(obj: torch.Tensor, starts: torch.Tensor, views: torch.Tensor) -> torch.Tensor:
    """In-place scatter-add of views (ObjectCutout.add, phaser/utils/object.py:540-557)."""
    S, H, W = _obj_dims(obj)
    B = starts.shape[0]
    views = views.contiguous()
    ny, nx = views.shape[-2:]
    name = {torch.complex64: 'phb_cutout_add_c64', torch.float32: 'phb_cutout_add_f32'}.get(obj.dtype)
    if name is None:
        raise TypeError(f"unsupported dtype {obj.dtype}")
    _lib.call(name, obj.data_ptr(), S, H, W, starts.data_ptr(), B, ny, nx, views.data_ptr(), _stream())
    return obj


def set_cutouts(obj: torch.Tensor, starts: torch.Tensor, views: torch.Tensor) -> torch.Tensor:
    """In-place overwrite of views (ObjectCutout.set, phaser/utils/object.py:521-538)."""
    if obj.dtype != torch.complex64:
        raise TypeError("set_cutouts supports complex64")
    S, H, W = _obj_dims(obj)
    views = views.contiguous()
    ny, nx = views.shape[-2:]
    _lib.call('phb_cutout_set_c64', obj.data_ptr(), S, H, W, starts.data_ptr(), starts.shape[0], ny, nx,
              views.data_ptr(), _stream())
    return obj
