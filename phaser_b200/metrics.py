"""Reconstruction-quality metrics on the device."""
from __future__ import annotations

import typing as t

import torch

from . import _lib


def object_nrmse(rec: torch.Tensor, ref: torch.Tensor, rows: t.Tuple[int, int], cols: t.Tuple[int, int]) -> float:
    """NRMSE of the projected object (product over slices) over rows x cols:
    linear phase ramps removed from both (least-squares planes,
    phb_remove_phase_ramp_c64), then the reconstruction's global phase fitted:
    |rec e^{i phi0} - ref| / |ref|."""
    pr = torch.prod(rec, dim=0, keepdim=True).contiguous()
    pt = torch.prod(ref, dim=0, keepdim=True).contiguous()
    sums = torch.zeros((1, 3), dtype=torch.float64, device=rec.device)
    H, W = pr.shape[-2:]
    st = torch.cuda.current_stream().cuda_stream
    for x in (pr, pt):
        _lib.call('phb_remove_phase_ramp_c64', x.data_ptr(), 1, H, W, rows[0], rows[1], cols[0], cols[1],
                  sums.data_ptr(), st)
    a = pr[0, rows[0]:rows[1], cols[0]:cols[1]].to(torch.complex128)
    b = pt[0, rows[0]:rows[1], cols[0]:cols[1]].to(torch.complex128)
    phi0 = torch.angle(torch.sum(torch.conj(a) * b))
    return float(torch.linalg.vector_norm(a * torch.exp(1j * phi0) - b) / torch.linalg.vector_norm(b))
