"""Data-parallel split of the engines over ranks (one process per GPU).

Every rank holds the whole reconstruction (object, probe, scan, patterns); each
mini-batch's positions are split into contiguous row ranges, one per rank.  A
rank runs the fused kernel on its rows only (PHB_FLAG_PARTIAL), the partial
accumulators -- object / illumination / probe sums (float32) and the
per-position and global step-size sums (float64) -- are summed over ranks
with one all-reduce each, and every rank then applies the identical update
(phb_solver_group_finish).  The iteration report (NaN status, error mean) is
combined the same way.  The reference runs one process; this split is the
mini-batch's one exchange step (the update reductions), so no other
communication is needed.

The gradient engine splits the same way: the object gradient (accumulated by
the kernel straight into the engine's gradient buffer), the probe-gradient
accumulator and the float64 loss / position sums are summed over ranks, then
every rank forms the identical gradients and applies the identical optimizer
step.  The group's NaN status is combined before anyone acts on it.
"""
from __future__ import annotations

import typing as t

import torch
import torch.distributed as dist

from .engines.conventional import ConventionalEngine
from .device import _ptr
from .engines.gradient import GradientEngine


def split_rows(B: int, world: int, rank: int) -> t.Tuple[int, int]:
    """Contiguous, balanced row range [b0, b1) of a B-row mini-batch for `rank`."""
    base, extra = divmod(B, world)
    b0 = rank * base + min(rank, extra)
    return b0, b0 + base + (1 if rank < extra else 0)


def allreduce_sum(tensors: t.Sequence[torch.Tensor], group=None) -> None:
    for x in tensors:
        dist.all_reduce(x, op=dist.ReduceOp.SUM, group=group)


def combine_report(report: torch.Tensor, group=None) -> None:
    """report = (status, n_outside, nanmean(errors), count) of this rank's rows ->
    the same over all ranks: status is the first group index that went non-finite
    (or -1), n_outside is identical on every rank, the mean is count-weighted."""
    status = report[0:1].clone()
    status[status < 0] = float('inf')
    dist.all_reduce(status, op=dist.ReduceOp.MIN, group=group)
    mc = torch.stack([torch.nan_to_num(report[2] * report[3], nan=0.0), report[3]])
    dist.all_reduce(mc, op=dist.ReduceOp.SUM, group=group)
    report[0] = torch.where(torch.isinf(status[0]), torch.full_like(status[0], -1.0), status[0])
    report[2] = torch.where(mc[1] > 0, mc[0] / mc[1], torch.full_like(mc[0], float('nan')))
    report[3] = mc[1]


class DistributedConventionalEngine(ConventionalEngine):
    """ConventionalEngine whose mini-batches are split over the ranks of `group`
    (torch.distributed, NCCL for GPUs).  Every rank must run the same iterations."""

    def __init__(self, args, props, *, group=None, **kw):
        super().__init__(args, props, **kw)
        self.pg = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        if self.eng.new_obj_mag is not None or self.eng.new_probe_mag is not None:
            raise NotImplementedError("illumination tracking is not split over ranks")
        self._views = self.eng.reduce_views()

    def _group_step(self, group: torch.Tensor, B: int, flags: int, gi: int, events, sched) -> None:
        eng = self.eng
        b0, b1 = split_rows(B, self.world, self.rank)
        f32, f64 = self._views
        if b1 > b0:
            eng.step(self.solver_kind, group, B, flags=flags, group_index=gi, events=events, rows=(b0, b1), **sched)
        else:   # no rows here: contribute zeros (the applies leave the other accumulators zeroed)
            f32.zero_()
            eng._last_step = eng._step_struct(self.solver_kind, flags, *self._sched_args(sched), gi, None, None,
                                              None, None, None, None, 1.0, None, (0, 1))
        allreduce_sum((f32, f64), self.pg)
        eng.finish(group, B)

    @staticmethod
    def _sched_args(sched):
        return (sched.get('beta_object', 1.0), sched.get('beta_probe', 1.0), sched.get('illum_reg_object', 1e-2),
                sched.get('illum_reg_probe', 1e-2), sched.get('gamma', 1e-4))

    def _combine_report(self, report: torch.Tensor) -> None:
        combine_report(report, self.pg)


def combine_status(status: torch.Tensor, group=None) -> None:
    """status (int32, -1 = fine, else the first bad group index) -> the minimum
    non-negative value over ranks, or -1 when every rank is fine."""
    big = torch.iinfo(torch.int32).max
    s = torch.where(status < 0, torch.full_like(status, big), status)
    dist.all_reduce(s, op=dist.ReduceOp.MIN, group=group)
    status.copy_(torch.where(s == big, torch.full_like(s, -1), s))


class DistributedGradientEngine(GradientEngine):
    """GradientEngine whose mini-batches are split over the ranks of `group`
    (torch.distributed, NCCL for GPUs).  Every rank must run the same iterations."""

    def __init__(self, args, props, *, group=None, **kw):
        super().__init__(args, props, **kw)
        self.pg = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self._views = self.eng.reduce_views()

    def _grad_step(self, group: torch.Tensor, B: int, flags: int, gi: int, events, iter_vars, group_loss,
                   probe_int: float) -> None:
        eng = self.eng
        b0, b1 = split_rows(B, self.world, self.rank)
        f32, f64 = self._views
        kw = self._grad_kw(B, iter_vars, group_loss, probe_int)
        if b1 > b0:
            eng.step('grad', group, B, flags=flags, group_index=gi, events=events, rows=(b0, b1), **kw)
        else:   # no rows here: contribute zeros (the applies leave the other accumulators zeroed,
            # and the engine zeroed the object gradient before this step)
            f32.zero_()
            st = eng._step_struct('grad', flags, 1.0, 1.0, 1e-2, 1e-2, 1e-4, gi, kw['grad_object'], kw['grad_probe'],
                                  kw['grad_pos'], None, None, None, kw['grad_pos_scale'], kw['group_loss'], (0, 1))
            st.grad_tilt, st.grad_tilt_scale = _ptr(kw['grad_tilt']), float(kw['grad_tilt_scale'])
            eng._last_step = st
        parts = [f32, f64] + ([kw['grad_object']] if kw['grad_object'] is not None else [])
        allreduce_sum(parts, self.pg)
        eng.finish(group, B)
        combine_status(eng.status, self.pg)

