"""The data-parallel mini-batch split on the GPU.  Only one GPU is available
here, so two ranks are emulated by two engines on the same device whose
partial steps never wait on each other: rank 1's accumulators are added into
rank 0's (what the all-reduce does), rank 0 finishes, and the result must
match one full step (1e-5 relative L2; fp32 atomics reorder sums).  A whole
run of DistributedConventionalEngine on a one-rank NCCL group must match
ConventionalEngine."""
import os
import socket

import numpy
import pytest
import torch
import torch.distributed as dist

from phaser_b200 import _lib
from phaser_b200 import plan as PL
from phaser_b200.distributed import DistributedConventionalEngine
from phaser_b200.engines.conventional import ConventionalEngine
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
