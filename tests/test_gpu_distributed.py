"""The data-parallel mini-batch split on the GPU.  Only one GPU is available
here, so two ranks are emulated by two engines on the same device whose
partial steps never wait on each other: rank 1's accumulators are added into
rank 0's (what the all-reduce does), rank 0 finishes, and the result must
match one full step (1e-5 relative L2; fp32 atomics reorder sums).  The same
holds for the gradient engine's loss and gradients, where the object gradient
buffer is summed too.  Whole runs of DistributedConventionalEngine and
DistributedGradientEngine on a one-rank NCCL group must match the plain
engines."""
import os
import socket

import numpy
import pytest
import torch
import torch.distributed as dist

from phaser_b200 import _lib
from phaser_b200 import plan as PL
from phaser_b200.distributed import DistributedConventionalEngine, DistributedGradientEngine
from phaser_b200.engines.conventional import ConventionalEngine
from phaser_b200.device import NoiseSpec
from phaser_b200.engines.gradient import GradientEngine
from phaser_b200.state import Patterns

from .cases import make_case
from .test_gpu_engine import engine_for, make_state, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('solver', ['lsqml', 'epie'])
def test_partial_steps_summed_match_one_step(solver):
    c = make_case(seed=71, N=64, M=2, S=3, scan_shape=(4, 4))
    idx = numpy.random.default_rng(2).permutation(16)[:11].astype(numpy.int64)
    flags = (_lib.PHB_FLAG_UPDATE_OBJECT | _lib.PHB_FLAG_UPDATE_PROBE | _lib.PHB_FLAG_UPDATE_POSITION
             | _lib.PHB_FLAG_CALC_ERROR)
    kw = dict(beta_object=0.9, beta_probe=0.8)
    full, r0, r1 = (engine_for(c, 11) for _ in range(3))
    outs = []
    for e in (full, r0, r1):
        e.status.fill_(-1)
        outs.append(e.group_tensor([idx])[0][0])
    full.step(solver, outs[0], 11, flags=flags, **kw)
    r0.step(solver, outs[1], 11, flags=flags, rows=(0, 5), **kw)
    r1.step(solver, outs[2], 11, flags=flags, rows=(5, 11), **kw)
    (a32, a64), (b32, b64) = r0.reduce_views(), r1.reduce_views()
    a32 += b32
    a64 += b64
    r0.finish(outs[1], 11)
    torch.cuda.synchronize()
    p_f, o_f, _ = full.host_state()
    p_0, o_0, _ = r0.host_state()
    assert rel_l2(o_0, o_f) < 1e-5
    assert rel_l2(p_0, p_f) < 1e-5
    assert rel_l2(r0.pos_update.cpu().numpy()[idx], full.pos_update.cpu().numpy()[idx]) < 1e-4
    err_f = full.errors.cpu().numpy()[idx]
    if solver == 'lsqml':
        # LSQ-ML's per-position errors are finished from the rank-summed float64 sums:
        # after finish every rank holds all of the group's errors
        err_s = r0.errors.cpu().numpy()[idx]
    else:   # ePIE writes each rank's rows' errors in its own step
        err_s = numpy.concatenate([r0.errors.cpu().numpy()[idx[:5]], r1.errors.cpu().numpy()[idx[5:]]])
    assert numpy.allclose(err_s, err_f, rtol=1e-5)
    assert int(r0.status.cpu()[0]) == -1


def test_distributed_engine_on_one_rank_matches_engine():
    c = make_case(seed=72, N=64, M=2, S=2, scan_shape=(5, 5))
    props = PL.ConventionalEnginePlan(
        noise_model={'type': 'amplitude', 'eps': 1e-2}, solver={'type': 'lsqml', 'gamma': 1e-3},
        position_solver={'type': 'momentum', 'step_size': 1e-2, 'max_step_size': 0.2}, niter=2, grouping=10,
        update_positions=True)
    args = dict(data=Patterns(c.patterns, c.mask), dtype=numpy.float32, seed='dist', recons_name='t')
    ref = ConventionalEngine(dict(args, state=make_state(c)), props)
    ref.presolve()
    errs_ref = [ref.iteration(i) for i in (1, 2)]
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('nccl', rank=0, world_size=1, device_id=torch.device('cuda', 0))
    try:
        eng = DistributedConventionalEngine(dict(args, state=make_state(c)), props)
        eng.presolve()
        errs = [eng.iteration(i) for i in (1, 2)]
        st_d, st_r = eng.finish(), ref.finish()
    finally:
        dist.destroy_process_group()
    assert numpy.allclose(errs, errs_ref, rtol=1e-5)
    assert rel_l2(st_d.object.data, st_r.object.data) < 1e-5
    assert rel_l2(st_d.probe.data, st_r.probe.data) < 1e-5
    assert numpy.max(numpy.abs(st_d.scan - st_r.scan)) < 1e-5


def test_partial_gradient_steps_summed_match_one_step():
    c = make_case(seed=73, N=64, M=2, S=3, scan_shape=(4, 4))
    idx = numpy.random.default_rng(3).permutation(16)[:11].astype(numpy.int64)
    flags = _lib.PHB_FLAG_UPDATE_OBJECT | _lib.PHB_FLAG_UPDATE_PROBE | _lib.PHB_FLAG_UPDATE_POSITION
    engs = [engine_for(c, 11, noise=NoiseSpec('poisson', 1e-3, 0.0, 0.1)) for _ in range(3)]
    bufs = []
    for e, rows in zip(engs, (None, (0, 4), (4, 11))):
        e.status.fill_(-1)
        g = e.group_tensor([idx])[0][0]
        b = dict(grad_object=torch.zeros_like(e.object), grad_probe=torch.zeros_like(e.probe),
                 grad_pos=torch.zeros_like(e.scan), group_loss=torch.zeros(1, dtype=torch.float64, device='cuda'))
        e.step('grad', g, 11, flags=flags, grad_pos_scale=-0.5, rows=rows, **b)
        bufs.append((g, b))
    (a32, a64), (b32, b64) = engs[1].reduce_views(), engs[2].reduce_views()
    a32 += b32
    a64 += b64
    bufs[1][1]['grad_object'] += bufs[2][1]['grad_object']
    engs[1].finish(bufs[1][0], 11)
    torch.cuda.synchronize()
    full, part = bufs[0][1], bufs[1][1]
    for k in ('grad_object', 'grad_probe'):
        assert rel_l2(part[k].cpu().numpy(), full[k].cpu().numpy()) < 1e-5, k
    assert rel_l2(part['grad_pos'].cpu().numpy()[idx], full['grad_pos'].cpu().numpy()[idx]) < 1e-4
    assert float(part['group_loss'][0]) == pytest.approx(float(full['group_loss'][0]), rel=1e-9)
    assert int(engs[1].status.cpu()[0]) == -1


def test_distributed_gradient_engine_on_one_rank_matches_engine():
    c = make_case(seed=74, N=64, M=2, S=2, scan_shape=(5, 5))
    props = PL.GradientEnginePlan(
        solvers={'object': {'type': 'adam', 'learning_rate': 1e-2}, 'probe': {'type': 'adam', 'learning_rate': 1e-3},
                 'positions': {'type': 'sgd', 'learning_rate': 1e-2}},
        noise_model={'type': 'poisson', 'eps': 1e-3}, niter=2, grouping=10, update_positions=True)
    args = dict(data=Patterns(c.patterns, c.mask), dtype=numpy.float32, seed='dist-grad', recons_name='t')
    ref = GradientEngine(dict(args, state=make_state(c)), props)
    ref.presolve()
    loss_ref = [ref.iteration(i) for i in (1, 2)]
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('nccl', rank=0, world_size=1, device_id=torch.device('cuda', 0))
    try:
        eng = DistributedGradientEngine(dict(args, state=make_state(c)), props)
        eng.presolve()
        loss = [eng.iteration(i) for i in (1, 2)]
        st_d, st_r = eng.finish(), ref.finish()
    finally:
        dist.destroy_process_group()
    assert numpy.allclose(loss, loss_ref, rtol=1e-5)
    assert rel_l2(st_d.object.data, st_r.object.data) < 1e-5
    assert rel_l2(st_d.probe.data, st_r.probe.data) < 1e-5
    assert numpy.max(numpy.abs(st_d.scan - st_r.scan)) < 1e-5
