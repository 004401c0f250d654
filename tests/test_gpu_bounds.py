"""The bounds-checking build of the library (libphaser_b200_bounds.so, loaded with
PHASER_B200_BOUNDS_CHECK=1; kernels compiled with -DPHB_BOUNDS_CHECK=1).

A group row outside [0, n_pos) reaches the kernels only through the C ABI (the
Python engine refuses it on the host, DeviceEngine.group_tensor): the test writes
one past the end and -1 into the uploaded group.  The bounds build skips those rows
before any access through them and reports PHB_STATUS_BOUNDS | group index in the
step's status; on valid groups it gives the default build's results.  Each case runs
in a child process, which loads the bounds build in place of the default one."""
import os
import subprocess
import sys

import numpy
import pytest
import torch

from phaser_b200 import _lib

from .cases import make_case
from .conftest import ROOT
from .test_gpu_engine import engine_for, rel_l2

pytestmark = pytest.mark.gpu

# LSQ-ML and the gradient engine (independent CTAs per (position, mode)), ePIE (one
# cluster of the modes per position) and N = 256 (one 4-CTA cluster per (position, mode))
CASES = {
    'lsqml-N64': ('lsqml', dict(seed=51, N=64, M=2, S=3)),
    'epie-N64': ('epie', dict(seed=52, N=64, M=2, S=2)),
    'grad-N64': ('grad', dict(seed=53, N=64, M=2, S=2)),
    'lsqml-N256': ('lsqml', dict(seed=54, N=256, M=2, S=2, scan_shape=(3, 3))),
}
GROUP_INDEX = 7


def run_step(eng, solver, group, B):
    """One mini-batch step with every update on; returns (status, object or its
    gradient, probe or its gradient) on the host."""
    eng.status.fill_(-1)
    upd = _lib.PHB_FLAG_UPDATE_OBJECT | _lib.PHB_FLAG_UPDATE_PROBE | _lib.PHB_FLAG_UPDATE_POSITION
    if solver == 'grad':
        g_obj, g_probe = torch.zeros_like(eng.object), torch.zeros_like(eng.probe)
        g_pos = torch.zeros_like(eng.scan)
        loss = torch.zeros((eng.n_pos,), dtype=torch.float32, device=eng.device)
        eng.step('grad', group, B, flags=upd, grad_object=g_obj, grad_probe=g_probe, grad_pos=g_pos, loss=loss,
                 group_index=GROUP_INDEX)
        obj, probe = g_obj.cpu().numpy(), g_probe.cpu().numpy()
    else:
        eng.step(solver, group, B, flags=upd | _lib.PHB_FLAG_CALC_ERROR, group_index=GROUP_INDEX)
        probe, obj, _ = eng.host_state()
    torch.cuda.synchronize()
    return int(eng.status.cpu()[0]), obj, probe


def case_group(c):
    n = c.scan.shape[0] * c.scan.shape[1]
    return numpy.arange(min(n, 8), dtype=numpy.int64)


def child(case: str, out: str) -> None:
    """Run in the child process (PHASER_B200_BOUNDS_CHECK=1): a valid group, then the same
    group on a fresh engine with rows 2 and 5 outside the scan."""
    lib = _lib.load()
    assert os.path.basename(lib._name) == 'libphaser_b200_bounds.so', lib._name
    solver, cfg = CASES[case]
    c = make_case(**cfg)
    idx = case_group(c)
    eng = engine_for(c, len(idx))
    gt, sizes = eng.group_tensor([idx])
    st_ok, obj_ok, probe_ok = run_step(eng, solver, gt[0], sizes[0])
    eng = engine_for(c, len(idx))
    gt, sizes = eng.group_tensor([idx])
    bad = gt[0].clone()
    bad[2] = eng.n_pos
    bad[5] = -1
    st_bad, obj_bad, probe_bad = run_step(eng, solver, bad, sizes[0])
    numpy.savez(out, st_ok=st_ok, obj_ok=obj_ok, probe_ok=probe_ok, st_bad=st_bad, obj_bad=obj_bad,
                probe_bad=probe_bad, obj0=c.obj, probe0=c.probe)


@pytest.mark.parametrize('case', list(CASES))
def test_bounds_build_skips_and_reports_rows_outside_the_scan(case, tmp_path):
    out = tmp_path / 'result.npz'
    env = dict(os.environ, PHASER_B200_BOUNDS_CHECK='1')
    code = f"from tests import test_gpu_bounds as T; T.child({case!r}, {str(out)!r})"
    subprocess.run([sys.executable, '-c', code], cwd=ROOT, env=env, check=True, timeout=900)
    r = numpy.load(out)
    assert int(r['st_ok']) == -1
    assert int(r['st_bad']) == _lib.PHB_STATUS_BOUNDS | GROUP_INDEX
    with pytest.raises(IndexError, match=f"group {GROUP_INDEX}"):
        _lib.raise_for_status(int(r['st_bad']))
    # the other rows ran: the update (or gradient) is finite and not zero
    assert numpy.isfinite(r['obj_bad']).all() and numpy.isfinite(r['probe_bad']).all()
    solver, cfg = CASES[case]
    if solver == 'grad':
        assert numpy.abs(r['obj_bad']).max() > 0
    else:
        assert rel_l2(r['obj_bad'], r['obj0']) > 1e-6
    # on a valid group the bounds build gives the default build's results (this process)
    assert os.path.basename(_lib.load()._name) == 'libphaser_b200.so'
    c = make_case(**cfg)
    idx = case_group(c)
    eng = engine_for(c, len(idx))
    gt, sizes = eng.group_tensor([idx])
    st, obj, probe = run_step(eng, solver, gt[0], sizes[0])
    assert st == -1
    assert rel_l2(r['obj_ok'], obj) < 1e-6
    assert rel_l2(r['probe_ok'], probe) < 1e-6
