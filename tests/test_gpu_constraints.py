"""GPU constraints and cost regularisers against the reference's own outputs
(tests/golden/constraints.npz) and the oracle.

Tolerances: the constraints within 1e-5 relative L2 of the reference's result
(complex64 logs / exponentials, float32 DFT sums over a whole slice); the cost
values within 1e-5 relative, their gradients within 1e-5 relative L2 of the
oracle's."""
import ctypes
import os
import types

import numpy
import pytest
import torch

from oracle import phaser_np as P
from phaser_b200 import _lib
from phaser_b200.constraints import build_constraints
from phaser_b200.engines.gradient import run_engine as run_gradient
from phaser_b200 import plan as PL
from phaser_b200.sampling import ObjectSampling
from phaser_b200.state import Patterns

from .cases import make_case
from .conftest import GOLDEN
from .test_gpu_engine import make_state, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def g():
    return dict(numpy.load(os.path.join(GOLDEN, 'constraints.npz'), allow_pickle=False))


def fake_engine(g):
    obj = torch.from_numpy(g['obj'].copy()).cuda()
    S, H, W = obj.shape
    osamp = ObjectSampling((H, W), g['obj_sampling'], g['corner'], g['region_min'], g['region_max'])
    state = types.SimpleNamespace(object=types.SimpleNamespace(thicknesses=g['thick']))
    return types.SimpleNamespace(object=obj, S=S, H=H, W=W, device=obj.device, obj_sampling=osamp), state


@pytest.mark.parametrize('hook,key', [
    ({'type': 'layers', 'sigma': 30.0, 'weight': 0.6}, 'layers'),
    ({'type': 'obj_low_pass', 'max_freq': 0.3}, 'low_pass'),
    ({'type': 'obj_gaussian', 'sigma': 0.7, 'weight': 0.8}, 'gaussian'),
    ({'type': 'remove_phase_ramp'}, 'phase_ramp'),
    ({'type': 'clamp_object_amplitude', 'amplitude': 1.1}, 'clamp'),
], ids=lambda v: v if isinstance(v, str) else v['type'])
def test_object_constraints_match_reference(g, hook, key):
    eng, state = fake_engine(g)
    (con,) = build_constraints([hook], eng, state, per_group=False)
    con.apply_iter()
    torch.cuda.synchronize()
    assert rel_l2(eng.object.cpu().numpy(), g[key]) < 1e-5


def test_layers_is_not_a_group_constraint(g):
    eng, state = fake_engine(g)
    with pytest.raises(ValueError):
        build_constraints([{'type': 'layers', 'sigma': 30.0}], eng, state, per_group=True)


def test_object_regularizers_match_oracle(g):
    costs = {'obj_l1': 0.3, 'obj_l2': 0.4, 'obj_phase_l1': 0.5, 'obj_tv': 0.6, 'obj_tikh': 0.7,
             'layers_tv': 0.8, 'layers_tikh': 0.9}
    reg = _lib.PhbObjReg(l1=0.3, l2=0.4, phase_l1=0.5, tikh=0.7, tv=0.6, tv_eps=1e-6, layers_tikh=0.9,
                         layers_tv=0.8, scale=0.25)
    obj = torch.from_numpy(g['obj']).cuda()
    S, H, W = obj.shape
    grad = torch.zeros_like(obj)
    loss = torch.zeros((1,), dtype=torch.float64, device='cuda')
    _lib.call('phb_object_regularizers', obj.data_ptr(), S, H, W, ctypes.byref(reg), grad.data_ptr(),
              loss.data_ptr(), torch.cuda.current_stream().cuda_stream)
    ref_cost, ref_grad = P.obj_regularizer_costs(g['obj'].astype(numpy.complex128), costs, 0.25, tv_eps=1e-6)
    assert float(loss.cpu()[0]) == pytest.approx(ref_cost, rel=1e-5)
    assert rel_l2(grad.cpu().numpy(), ref_grad) < 1e-5


def test_gradient_run_with_regularizers_matches_oracle():
    c = make_case(seed=93, N=64, M=2, S=2, scan_shape=(5, 5))
    regs = {'obj_l2': 0.01, 'obj_tikh': 0.005, 'layers_tikh': 0.05}
    props = PL.GradientEnginePlan(
        solvers={'object': {'type': 'sgd', 'learning_rate': 2.0, 'momentum': 0.5},
                 'probe': {'type': 'adam', 'learning_rate': 1e-3}},
        regularizers=[{'type': k, 'cost': v} for (k, v) in regs.items()],
        noise_model={'type': 'poisson', 'eps': 1e-3}, niter=3, grouping=10)
    state = run_gradient({'data': Patterns(c.patterns, c.mask), 'state': make_state(c), 'dtype': numpy.float32,
                          'seed': 'reg-seed', 'recons_name': 't'}, props)
    run = P.GradientRun(solvers={('object',): ('sgd', dict(learning_rate=2.0, momentum=0.5)),
                                 ('probe',): ('adam', dict(learning_rate=1e-3))},
                        niter=3, grouping=10, seed='reg-seed', noise=P.NoiseModel(kind='poisson', eps=1e-3),
                        regularizers=regs)
    probe, obj, scan, losses = P.run_gradient(
        run, probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
        probe_sampling=c.probe_sampling, corner=c.osamp.corner, obj_sampling=c.osamp.sampling,
        thicknesses=c.thick, wavelength=c.wavelength)
    assert numpy.allclose(state.progress.detector_errors, losses, rtol=1e-4)
    assert rel_l2(state.object.data, obj) < 1e-4
    assert rel_l2(state.object.data - c.obj, obj - c.obj) < 1e-2
    assert rel_l2(state.probe.data, probe) < 1e-4


def test_probe_and_recip_regularizers_match_oracle(g):
    rng = numpy.random.default_rng(12)
    probe = (rng.normal(size=(2, 64, 64)) + 1j * rng.normal(size=(2, 64, 64))).astype(numpy.complex64)
    pd = torch.from_numpy(probe).cuda()
    costs = {'probe_phase_tikh': 0.02, 'probe_recip_tikh': 0.03, 'probe_recip_tv': 0.04}
    reg = _lib.PhbProbeReg(phase_tikh=0.02, recip_tikh=0.03, recip_tv=0.04, tv_eps=1e-6)
    scratch = torch.empty((2 * 2 * 64 * 64,), dtype=torch.complex64, device='cuda')
    grad = torch.zeros_like(pd)
    loss = torch.zeros((1,), dtype=torch.float64, device='cuda')
    _lib.call('phb_probe_regularizers', pd.data_ptr(), 2, 64, ctypes.byref(reg), grad.data_ptr(), loss.data_ptr(),
              scratch.data_ptr(), torch.cuda.current_stream().cuda_stream)
    ref_cost, ref_grad = P.probe_regularizer_costs(probe.astype(numpy.complex128), costs, tv_eps=1e-6)
    assert float(loss.cpu()[0]) == pytest.approx(ref_cost, rel=1e-4)
    assert rel_l2(grad.cpu().numpy(), ref_grad) < 1e-4
    # object: sum |fft2(prod O)| on an odd-sized grid
    obj = torch.from_numpy(g['obj']).cuda()
    S, H, W = obj.shape
    scr = torch.empty(((2 + S) * H * W,), dtype=torch.complex64, device='cuda')
    grad = torch.zeros_like(obj)
    loss.zero_()
    _lib.call('phb_object_recip_l1', obj.data_ptr(), S, H, W, 0.01 * 0.25, grad.data_ptr(), loss.data_ptr(),
              scr.data_ptr(), torch.cuda.current_stream().cuda_stream)
    ref_cost, ref_grad = P.obj_recip_l1(g['obj'].astype(numpy.complex128), 0.01, 0.25)
    assert float(loss.cpu()[0]) == pytest.approx(ref_cost, rel=1e-5)
    assert rel_l2(grad.cpu().numpy(), ref_grad) < 1e-4


def test_gradient_run_with_fourier_regularizers_matches_oracle():
    c = make_case(seed=94, N=64, M=2, S=2, scan_shape=(5, 5))
    regs = {'obj_recip_l1': 1e-3, 'probe_recip_tikh': 1e-4, 'probe_recip_tv': 1e-4}
    props = PL.GradientEnginePlan(
        solvers={'object': {'type': 'sgd', 'learning_rate': 2.0, 'momentum': 0.5},
                 'probe': {'type': 'adam', 'learning_rate': 1e-3}},
        regularizers=[{'type': k, 'cost': v} for (k, v) in regs.items()],
        noise_model={'type': 'poisson', 'eps': 1e-3}, niter=3, grouping=10)
    state = run_gradient({'data': Patterns(c.patterns, c.mask), 'state': make_state(c), 'dtype': numpy.float32,
                          'seed': 'reg-seed', 'recons_name': 't'}, props)
    run = P.GradientRun(solvers={('object',): ('sgd', dict(learning_rate=2.0, momentum=0.5)),
                                 ('probe',): ('adam', dict(learning_rate=1e-3))},
                        niter=3, grouping=10, seed='reg-seed', noise=P.NoiseModel(kind='poisson', eps=1e-3),
                        regularizers=regs)
    probe, obj, scan, losses = P.run_gradient(
        run, probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
        probe_sampling=c.probe_sampling, corner=c.osamp.corner, obj_sampling=c.osamp.sampling,
        thicknesses=c.thick, wavelength=c.wavelength)
    assert numpy.allclose(state.progress.detector_errors, losses, rtol=1e-4)
    assert rel_l2(state.object.data, obj) < 1e-4
    assert rel_l2(state.probe.data, probe) < 1e-4


def test_tilt_gaussian_matches_reference(g):
    eng, state = fake_engine(g)
    eng.tilt = torch.from_numpy(g['tilt_in'].reshape(-1, 2).astype(numpy.float32)).cuda()
    eng.scan = torch.from_numpy(g['scan'].reshape(-1, 2).astype(numpy.float32)).cuda()
    eng.n_pos = eng.scan.shape[0]
    (con,) = build_constraints([{'type': 'tilt_gaussian', 'sigma': 0.8, 'weight': 0.7}], eng, state, per_group=False)
    con.apply_iter()
    out = eng.tilt.cpu().numpy().reshape(g['tilt_gaussian'].shape)
    assert numpy.max(numpy.abs(out - g['tilt_gaussian'])) < 1e-5 * numpy.max(numpy.abs(g['tilt_gaussian']))
