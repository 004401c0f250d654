"""The multislice forward model as a differentiable torch function.

`multislice_loss(obj, probe, scan, engine, group, B)` returns the gradient
engine's data loss of one mini-batch (the noise model's summed loss,
phaser/engines/gradient/run.py:357-405) as a float64 scalar tensor; its
gradients with respect to the object (S, H, W), probe modes (M, N, N) and scan
positions (P, 2) come from the hand-written adjoint of the fused kernel, which
replaces jax.value_and_grad.  The kernel evaluates loss and adjoint in one
launch, so the forward pass already holds the gradients and the backward pass
only scales them by the incoming gradient.  Every slice's incident wavefield
is kept (the per-slice checkpoints) in the engine's workspace for the adjoint:
B_max x M x S x N^2 complex values, bounded by the group size.  From them the
adjoint recomputes each slice's transmitted wave, its propagation and the
object cutouts; no other forward intermediate is stored.

Complex gradients follow torch's convention, dL/dRe + i dL/dIm, so
`obj.grad` is what torch.autograd gives for a real loss of a complex leaf;
phaser's descent direction is its negative.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .device import DeviceEngine


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class MultisliceLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, obj: torch.Tensor, probe: torch.Tensor, scan: torch.Tensor, engine: DeviceEngine,
                group: torch.Tensor, B: int) -> torch.Tensor:
        eng = engine
        for name, x, shape, dt in (('object', obj, (eng.S, eng.H, eng.W), torch.complex64),
                                   ('probe', probe, (eng.M, eng.N, eng.N), torch.complex64),
                                   ('scan', scan, (eng.n_pos, 2), torch.float32)):
            if tuple(x.shape) != shape or x.dtype != dt or not x.is_contiguous() or x.device != eng.object.device:
                raise ValueError(f"{name} must be a contiguous {dt} tensor of shape {shape} on {eng.object.device}")
        desc = _lib.PhbEngine.from_buffer_copy(eng.desc)
        desc.object, desc.probe, desc.scan = obj.data_ptr(), probe.data_ptr(), scan.data_ptr()
        dref = ctypes.byref(desc)
        # the workspace caches the probe's spectrum: refresh it for this probe
        _lib.call('phb_engine_probe_changed', dref, _stream())
        need_o, need_p, need_s = ctx.needs_input_grad[:3]
        g_obj = torch.zeros_like(obj) if need_o else None
        g_probe = torch.zeros_like(probe) if need_p else None
        g_pos = torch.zeros_like(scan) if need_s else None
        loss = torch.zeros((1,), dtype=torch.float64, device=eng.device)
        st = _lib.PhbStep()
        st.solver = _lib.PHB_SOLVER_GRAD
        st.flags = ((_lib.PHB_FLAG_UPDATE_OBJECT if need_o else 0) | (_lib.PHB_FLAG_UPDATE_PROBE if need_p else 0)
                    | (_lib.PHB_FLAG_UPDATE_POSITION if need_s else 0))
        st.grad_object = 0 if g_obj is None else g_obj.data_ptr()
        st.grad_probe = 0 if g_probe is None else g_probe.data_ptr()
        st.grad_pos = 0 if g_pos is None else g_pos.data_ptr()
        st.grad_pos_scale = 1.0
        st.group_loss = loss.data_ptr()
        st.pos_update, st.errors = eng.pos_update.data_ptr(), eng.errors.data_ptr()
        eng.status.fill_(-1)
        st.status, st.group_index = eng.status.data_ptr(), 0
        _lib.call('phb_solver_group', dref, ctypes.byref(st), group.data_ptr(), int(B), _stream())
        ctx.save_for_backward(*(x for x in (g_obj, g_probe, g_pos) if x is not None))
        ctx.which = (need_o, need_p, need_s)
        ctx.status = eng.status
        return loss[0]

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        status = int(ctx.status.cpu()[0])
        if status >= _lib.PHB_STATUS_BOUNDS:   # an aborted kernel, or a position outside the scan
            _lib.raise_for_status(status)
        saved = list(ctx.saved_tensors)
        out = []
        for need in ctx.which:
            out.append(saved.pop(0) * grad_out.to(torch.float32) if need else None)
        return (*out, None, None, None)


def multislice_loss(obj: torch.Tensor, probe: torch.Tensor, scan: torch.Tensor, engine: DeviceEngine,
                    group: torch.Tensor, B: int) -> torch.Tensor:
    """Summed noise-model loss of the B positions `group` (device int64), differentiable
    with respect to `obj`, `probe` and `scan`."""
    return MultisliceLoss.apply(obj, probe, scan, engine, group, B)
