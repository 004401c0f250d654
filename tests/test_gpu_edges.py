"""Edge cases of the fused kernel against the oracle: cutouts that hang past the
object's edge (out-of-bounds pixels read as transmission 1 and are not
scattered), the largest mode count (8 modes: a cluster of 8 CTAs), many
slices, single-position groups.  Tolerances as in test_gpu_engine.py /
test_gpu_gradient.py."""
import numpy
import pytest
import torch

from oracle import phaser_np as P
from phaser_b200 import _lib

from .cases import make_case
from .test_gpu_engine import rel_l2, run_group
from .test_gpu_gradient import NOISES
from phaser_b200.device import DeviceEngine

pytestmark = pytest.mark.gpu

EDGE_CONFIGS = [
    ('lsqml', dict(seed=111, N=64, M=2, S=3, pad_px=-14.0)),
    ('epie', dict(seed=112, N=64, M=2, S=2, pad_px=-14.0)),
    ('lsqml', dict(seed=113, N=128, M=8, S=2, scan_shape=(3, 3))),
    ('epie', dict(seed=114, N=128, M=8, S=2, scan_shape=(3, 3))),
    ('lsqml', dict(seed=115, N=128, M=2, S=16, scan_shape=(2, 2))),
    ('lsqml', dict(seed=116, N=64, M=8, S=3, scan_shape=(3, 3))),
]


@pytest.mark.parametrize('solver,cfg', EDGE_CONFIGS,
                         ids=[f"{s}-N{c['N']}M{c['M']}S{c['S']}{'-edge' if c.get('pad_px') else ''}"
                              for s, c in EDGE_CONFIGS])
def test_group_step_edge_cases_match_oracle(solver, cfg):
    c = make_case(**cfg)
    if cfg.get('pad_px'):   # the case really has cutouts past the edge
        g = c.geom()
        starts = P.cutout_starts(c.scan.reshape(-1, 2), g.corner, g.obj_sampling, c.probe.shape[-2:])
        H, W = c.obj.shape[-2:]
        assert (starts.min() < 0) or (starts[:, 0].max() + c.probe.shape[-1] > H)
    params = (P.LSQMLParams(0.9, 0.8, 1e-2, 1e-2, 1e-4) if solver == 'lsqml' else P.EPIEParams(0.7, 0.6))
    got, ref = run_group(c, solver, dict(update_position=True), params)
    assert rel_l2(got['obj'], ref['object']) < 1e-5
    assert rel_l2(got['probe'], ref['probe']) < 1e-5
    assert rel_l2(got['obj'] - c.obj, ref['object'] - c.obj) < 1e-3
    assert numpy.allclose(got['errors'], ref['errors'], rtol=1e-4)
    assert rel_l2(got['pos'], ref['pos_update']) < 2e-3


@pytest.mark.parametrize('cfg', [dict(seed=117, N=64, M=2, S=3, pad_px=-14.0),
                                 dict(seed=118, N=128, M=2, S=16, scan_shape=(2, 2)),
                                 dict(seed=119, N=128, M=8, S=2, scan_shape=(2, 2))],
                         ids=['edge', 'S16', 'M8'])
def test_gradient_edge_cases_match_oracle(cfg):
    c = make_case(**cfg)
    n = c.scan.shape[0] * c.scan.shape[1]
    idx = numpy.arange(n, dtype=numpy.int64)
    onoise, spec = NOISES['poisson']
    eng = DeviceEngine(probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
                       probe_sampling=c.probe_sampling, obj_sampling=c.osamp, thicknesses=c.thick,
                       wavelength=c.wavelength, noise=spec, group_max=n)
    gt, sizes = eng.group_tensor([idx])
    g_obj, g_probe, g_pos = torch.zeros_like(eng.object), torch.zeros_like(eng.probe), torch.zeros_like(eng.scan)
    loss = torch.zeros((1,), dtype=torch.float64, device='cuda')
    eng.status.fill_(-1)
    eng.step('grad', gt[0], sizes[0], flags=_lib.PHB_FLAG_UPDATE_OBJECT | _lib.PHB_FLAG_UPDATE_PROBE
             | _lib.PHB_FLAG_UPDATE_POSITION, grad_object=g_obj, grad_probe=g_probe, grad_pos=g_pos, group_loss=loss)
    torch.cuda.synchronize()
    assert int(eng.status.cpu()[0]) == -1
    L, r_obj, r_probe, r_pos = P.grad_model_grads(
        c.geom(), c.probe, c.obj, c.scan.reshape(-1, 2), c.patterns.reshape(-1, *c.probe.shape[-2:]), c.mask,
        c.props(), None, onoise)
    assert float(loss.cpu()[0]) == pytest.approx(float(L), rel=1e-5)
    assert rel_l2(g_obj.cpu().numpy(), r_obj) < 1e-4
    assert rel_l2(g_probe.cpu().numpy(), r_probe) < 1e-4
    assert rel_l2(g_pos.cpu().numpy(), r_pos) < 1e-3


def test_single_position_group():
    c = make_case(seed=120, N=128, M=4, S=2, scan_shape=(1, 1))
    got, ref = run_group(c, 'lsqml', dict(update_position=True), P.LSQMLParams(0.9, 0.8, 1e-2, 1e-2, 1e-4))
    assert rel_l2(got['obj'], ref['object']) < 1e-5
    assert rel_l2(got['probe'], ref['probe']) < 1e-5
