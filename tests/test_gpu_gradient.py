"""GPU parity of the gradient engine against the numpy oracle.

- one mini-batch of the fused kernel in gradient mode (loss and hand-written
  adjoint) against the oracle's adjoint (itself checked against float64 central
  finite differences by test_oracle_gradient.py): loss within 1e-5 relative,
  object / probe gradients within 1e-4 relative L2, position gradients within
  1e-3 (a sum of products of float32 fields over the whole cutout);
- the optax-semantics update kernels against the oracle's restatement over
  three steps: within 1e-5 relative L2 of the oracle's parameters;
- whole runs of run_engine against the oracle's gradient-engine loop: object,
  probe and positions within 1e-4 after three iterations, loss history within
  1e-4 relative."""
import ctypes

import numpy
import pytest
import torch

from oracle import phaser_np as P
from phaser_b200 import _lib
from phaser_b200 import plan as PL
from phaser_b200.device import DeviceEngine, NoiseSpec
from phaser_b200.engines.gradient import DeviceSolver, run_engine
from phaser_b200.state import Patterns

from .cases import make_case
from .test_gpu_engine import make_state, rel_l2

pytestmark = pytest.mark.gpu

NOISES = {
    'amplitude': (P.NoiseModel(eps=1e-2), NoiseSpec('amplitude', 1e-2, 0.0, 0.1)),
    'anscombe': (P.NoiseModel.anscombe(eps=1e-2), NoiseSpec('anscombe', 1e-2, 0.375, 0.1)),
    'poisson': (P.NoiseModel(kind='poisson', eps=1e-3), NoiseSpec('poisson', 1e-3, 0.0, 0.1)),
}

GRAD_CONFIGS = [
    ('amplitude', dict(seed=81, N=64, M=2, S=3)),
    ('poisson', dict(seed=82, N=64, M=1, S=2)),
    ('anscombe', dict(seed=83, N=128, M=4, S=2)),
    ('amplitude', dict(seed=84, N=64, M=2, S=2, tilt=True)),
    ('poisson', dict(seed=85, N=128, M=2, S=5, scan_shape=(3, 3))),
    ('poisson', dict(seed=86, N=256, M=2, S=3, scan_shape=(2, 2))),
    ('amplitude', dict(seed=87, N=256, M=2, S=2, scan_shape=(2, 2), tilt=True)),
]


@pytest.mark.parametrize('noise,cfg', GRAD_CONFIGS,
                         ids=[f"{n}-N{c['N']}M{c['M']}S{c['S']}-{i}" for i, (n, c) in enumerate(GRAD_CONFIGS)])
def test_grad_step_matches_oracle_adjoint(noise, cfg):
    c = make_case(**cfg)
    n = c.scan.shape[0] * c.scan.shape[1]
    rng = numpy.random.default_rng(7)
    idx = rng.permutation(n)[: max(2, (2 * n) // 3)].astype(numpy.int64)
    onoise, spec = NOISES[noise]
    eng = DeviceEngine(probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
                       probe_sampling=c.probe_sampling, obj_sampling=c.osamp, thicknesses=c.thick,
                       wavelength=c.wavelength, tilt=c.tilt, noise=spec, group_max=len(idx))
    gt, sizes = eng.group_tensor([idx])
    g_obj = torch.zeros_like(eng.object)
    g_probe = torch.zeros_like(eng.probe)
    g_pos = torch.zeros_like(eng.scan)
    loss = torch.zeros((n,), dtype=torch.float32, device=eng.device)
    total = torch.zeros((1,), dtype=torch.float64, device=eng.device)
    flags = _lib.PHB_FLAG_UPDATE_OBJECT | _lib.PHB_FLAG_UPDATE_PROBE | _lib.PHB_FLAG_UPDATE_POSITION
    eng.status.fill_(-1)
    eng.step('grad', gt[0], sizes[0], flags=flags, grad_object=g_obj, grad_probe=g_probe, grad_pos=g_pos,
             loss=loss, group_loss=total)
    torch.cuda.synchronize()
    assert int(eng.status.cpu()[0]) == -1
    g = c.geom()
    tl = None if c.tilt is None else c.tilt.reshape(-1, 2)[idx]
    L, r_obj, r_probe, r_pos = P.grad_model_grads(
        g, c.probe, c.obj, c.scan.reshape(-1, 2)[idx], c.patterns.reshape(-1, *c.probe.shape[-2:])[idx],
        c.mask, c.props(), tl, onoise)
    assert float(total.cpu()[0]) == pytest.approx(float(L), rel=1e-5)
    assert float(loss.cpu().numpy()[idx].astype(numpy.float64).sum()) == pytest.approx(float(L), rel=1e-5)
    assert rel_l2(g_obj.cpu().numpy(), r_obj) < 1e-4
    assert rel_l2(g_probe.cpu().numpy(), r_probe) < 1e-4
    assert rel_l2(g_pos.cpu().numpy()[idx], r_pos) < 1e-3


OPTIMS = [
    ('sgd', dict(learning_rate=0.3)),
    ('sgd', dict(learning_rate=0.3, momentum=0.8, nesterov=True)),
    ('sgd', dict(learning_rate=0.3, momentum=0.8, nesterov=False)),
    ('adam', dict(learning_rate=1e-2)),
    ('adam', dict(learning_rate=1e-2, b1=0.8, b2=0.99, eps=1e-6, eps_root=1e-9, nesterov=True)),
    ('polyak_sgd', dict(max_learning_rate=2.0, f_min=0.1, scaling=0.5, eps=1e-3)),
]


@pytest.mark.parametrize('kind,props', OPTIMS, ids=[f"{k}-{i}" for i, (k, _) in enumerate(OPTIMS)])
def test_optimizer_kernels_match_oracle(kind, props):
    rng = numpy.random.default_rng(3)
    obj = (rng.normal(size=(2, 37, 41)) + 1j * rng.normal(size=(2, 37, 41))).astype(numpy.complex64)
    pos = rng.normal(size=(53, 2)).astype(numpy.float32)
    params = {'object': torch.from_numpy(obj.copy()).cuda(), 'positions': torch.from_numpy(pos.copy()).cuda()}
    sol = DeviceSolver(kind, dict(props), params)
    sol.update_for_iter({})
    ref = P.OptaxNP(kind, props, {'object': obj, 'positions': pos})
    status = torch.full((1,), -1, dtype=torch.int32, device='cuda')
    loss = torch.zeros((1,), dtype=torch.float64, device='cuda')
    scales = {'object': -0.25, 'positions': 2.0}
    for step in range(3):
        g_obj = (rng.normal(size=obj.shape) + 1j * rng.normal(size=obj.shape)).astype(numpy.complex64)
        g_pos = rng.normal(size=pos.shape).astype(numpy.float32)
        L = float(rng.uniform(1.0, 3.0))
        loss.fill_(L)
        sol.update(params, {'object': (torch.from_numpy(g_obj).cuda(), scales['object']),
                            'positions': (torch.from_numpy(g_pos).cuda(), scales['positions'])},
                   loss, status=status, status_code=step)
        upd = ref.update({'object': (scales['object'] * g_obj).astype(numpy.complex64),
                          'positions': (scales['positions'] * g_pos).astype(numpy.float32)}, L)
        obj = obj + upd['object']
        pos = pos + upd['positions']
        torch.cuda.synchronize()
        assert rel_l2(params['object'].cpu().numpy(), obj) < 1e-5
        assert rel_l2(params['positions'].cpu().numpy(), pos) < 1e-5
    assert int(status.cpu()[0]) == -1


def test_optimizer_flags_nonfinite_parameters():
    p = torch.ones((64,), dtype=torch.complex64, device='cuda')
    g = torch.zeros((64,), dtype=torch.complex64, device='cuda')
    g[17] = float('nan')
    sol = DeviceSolver('sgd', {'learning_rate': 1.0}, {'object': p})
    sol.update_for_iter({})
    status = torch.full((1,), -1, dtype=torch.int32, device='cuda')
    sol.update({'object': p}, {'object': (g, 1.0)}, torch.zeros((1,), dtype=torch.float64, device='cuda'),
               status=status, status_code=5)
    assert int(status.cpu()[0]) == 5


def test_add_centred_subtracts_the_mean_update():
    rng = numpy.random.default_rng(4)
    scan = rng.normal(size=(3000, 2)).astype(numpy.float32)
    upd = rng.normal(size=(3000, 2)).astype(numpy.float32)
    s = torch.from_numpy(scan.copy()).cuda()
    _lib.call('phb_add_centred', s.data_ptr(), torch.from_numpy(upd).cuda().data_ptr(), 3000,
              torch.cuda.current_stream().cuda_stream)
    ref = scan + (upd - upd.astype(numpy.float64).mean(axis=0))
    assert numpy.max(numpy.abs(s.cpu().numpy() - ref)) < 1e-6


RUNS = [
    ('sgd-momentum/polyak/adam', {
        'object': ('sgd', dict(learning_rate=20.0, momentum=0.5)),
        'probe': ('polyak_sgd', dict(max_learning_rate=1.0, f_min=0.0, scaling=0.1)),
        'positions': ('adam', dict(learning_rate=1e-2)),
    }, 'amplitude'),
    ('joint sgd/sgd', {
        ('object', 'probe'): ('sgd', dict(learning_rate=1.0)),
        'positions': ('sgd', dict(learning_rate=5.0, momentum=0.5, nesterov=False)),
    }, 'poisson'),
]


@pytest.mark.parametrize('name,solvers,noise', RUNS, ids=[r[0] for r in RUNS])
def test_run_engine_matches_oracle_gradient_loop(name, solvers, noise):
    c = make_case(seed=91, N=64, M=2, S=2, scan_shape=(5, 5))
    onoise, spec = NOISES[noise]
    plan_solvers = {(k if isinstance(k, str) else ','.join(k)): dict(type=kind, **sp)
                    for (k, (kind, sp)) in solvers.items()}
    noise_hook = {'type': noise, 'eps': onoise.eps}
    props = PL.GradientEnginePlan(solvers=plan_solvers, noise_model=noise_hook, niter=3, grouping=10,
                                  update_positions=True)
    state = run_engine({'data': Patterns(c.patterns, c.mask), 'state': make_state(c), 'dtype': numpy.float32,
                        'seed': 'grad-seed', 'recons_name': 't'}, props)
    run = P.GradientRun(solvers={((k,) if isinstance(k, str) else k): v for (k, v) in solvers.items()},
                        niter=3, grouping=10, seed='grad-seed', noise=onoise, update_positions=True)
    probe, obj, scan, losses = P.run_gradient(
        run, probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
        probe_sampling=c.probe_sampling, corner=c.osamp.corner, obj_sampling=c.osamp.sampling,
        thicknesses=c.thick, wavelength=c.wavelength)
    assert numpy.allclose(state.progress.detector_errors, losses, rtol=1e-4)
    assert rel_l2(state.object.data, obj) < 1e-4
    assert rel_l2(state.probe.data, probe) < 1e-4
    assert rel_l2(state.object.data - c.obj, obj - c.obj) < 1e-2
    assert numpy.max(numpy.abs(state.scan - scan)) < 1e-4


def test_run_engine_matches_oracle_gradient_loop_n256():
    """Two gradient-engine iterations at a 256^2 probe and detector: Adam on object and
    probe, SGD on positions, Poisson noise model."""
    c = make_case(seed=92, N=256, M=2, S=2, scan_shape=(3, 3))
    solvers = {'object': ('adam', dict(learning_rate=1e-2)), 'probe': ('adam', dict(learning_rate=1e-3)),
               'positions': ('sgd', dict(learning_rate=5.0, momentum=0.5, nesterov=False))}
    onoise, _ = NOISES['poisson']
    props = PL.GradientEnginePlan(solvers={k: dict(type=kind, **sp) for (k, (kind, sp)) in solvers.items()},
                                  noise_model={'type': 'poisson', 'eps': onoise.eps}, niter=2, grouping=5,
                                  update_positions=True)
    state = run_engine({'data': Patterns(c.patterns, c.mask), 'state': make_state(c), 'dtype': numpy.float32,
                        'seed': 'grad-seed-256', 'recons_name': 't'}, props)
    run = P.GradientRun(solvers={(k,): v for (k, v) in solvers.items()}, niter=2, grouping=5, seed='grad-seed-256',
                        noise=onoise, update_positions=True)
    probe, obj, scan, losses = P.run_gradient(
        run, probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
        probe_sampling=c.probe_sampling, corner=c.osamp.corner, obj_sampling=c.osamp.sampling,
        thicknesses=c.thick, wavelength=c.wavelength)
    assert numpy.allclose(state.progress.detector_errors, losses, rtol=1e-4)
    assert rel_l2(state.object.data, obj) < 1e-4
    assert rel_l2(state.probe.data, probe) < 1e-4
    assert numpy.max(numpy.abs(state.scan - scan)) < 1e-4


def test_positions_leaving_the_object_raise_value_error():
    """A position step that throws the probe off the object ends the run with the
    reference's error (utils/object.py:288-289), counted on the device."""
    c = make_case(seed=93, N=64, M=1, S=1, scan_shape=(4, 4))
    props = PL.GradientEnginePlan(
        solvers={'object': {'type': 'sgd', 'learning_rate': 1.0}, 'positions': {'type': 'sgd', 'learning_rate': 1e9}},
        noise_model={'type': 'amplitude'}, niter=2, grouping=8, update_positions=True)
    with pytest.raises(ValueError, match='probe positions completely outside object'):
        run_engine({'data': Patterns(c.patterns, c.mask), 'state': make_state(c), 'dtype': numpy.float32,
                    'seed': 'outside', 'recons_name': 't'}, props)


def test_autograd_function_matches_oracle_adjoint():
    """torch.autograd through the hand-written adjoint: loss, and the gradients of
    2 * loss with respect to object, probe and scan, against the oracle."""
    from phaser_b200.autograd import multislice_loss
    c = make_case(seed=86, N=64, M=2, S=3)
    n = c.scan.shape[0] * c.scan.shape[1]
    idx = numpy.random.default_rng(8).permutation(n)[: (2 * n) // 3].astype(numpy.int64)
    onoise, spec = NOISES['amplitude']
    eng = DeviceEngine(probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
                       probe_sampling=c.probe_sampling, obj_sampling=c.osamp, thicknesses=c.thick,
                       wavelength=c.wavelength, noise=spec, group_max=len(idx))
    gt, sizes = eng.group_tensor([idx])
    obj = eng.object.clone().requires_grad_()
    probe = eng.probe.clone().requires_grad_()
    scan = eng.scan.clone().requires_grad_()
    loss = multislice_loss(obj, probe, scan, eng, gt[0], sizes[0])
    (2.0 * loss).backward()
    loss = loss.detach()
    L, r_obj, r_probe, r_pos = P.grad_model_grads(
        c.geom(), c.probe, c.obj, c.scan.reshape(-1, 2)[idx], c.patterns.reshape(-1, 64, 64)[idx],
        c.mask, c.props(), None, onoise)
    assert float(loss) == pytest.approx(float(L), rel=1e-5)
    assert rel_l2(obj.grad.cpu().numpy(), 2 * r_obj) < 1e-4
    assert rel_l2(probe.grad.cpu().numpy(), 2 * r_probe) < 1e-4
    assert rel_l2(scan.grad.cpu().numpy()[idx], 2 * r_pos) < 1e-3
    # only the object: no probe / position adjoint requested
    obj2 = eng.object.clone().requires_grad_()
    (g,) = torch.autograd.grad(multislice_loss(obj2, eng.probe, eng.scan, eng, gt[0], sizes[0]), (obj2,))
    assert rel_l2(g.cpu().numpy(), r_obj) < 1e-4


@pytest.mark.parametrize('cfg', [dict(seed=87, N=64, M=2, S=3), dict(seed=88, N=128, M=2, S=4, scan_shape=(3, 3)),
                                 dict(seed=89, N=256, M=2, S=3, scan_shape=(2, 2))],
                         ids=['N64M2S3', 'N128M2S4', 'N256M2S3'])
def test_tilt_gradient_matches_oracle_adjoint(cfg):
    c = make_case(tilt=True, **cfg)
    n = c.scan.shape[0] * c.scan.shape[1]
    idx = numpy.random.default_rng(9).permutation(n)[: max(2, (2 * n) // 3)].astype(numpy.int64)
    onoise, spec = NOISES['poisson']
    eng = DeviceEngine(probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
                       probe_sampling=c.probe_sampling, obj_sampling=c.osamp, thicknesses=c.thick,
                       wavelength=c.wavelength, tilt=c.tilt, noise=spec, group_max=len(idx))
    gt, sizes = eng.group_tensor([idx])
    g_tilt = torch.zeros_like(eng.scan)
    loss = torch.zeros((1,), dtype=torch.float64, device='cuda')
    eng.status.fill_(-1)
    eng.step('grad', gt[0], sizes[0], flags=_lib.PHB_FLAG_UPDATE_TILT, grad_tilt=g_tilt, group_loss=loss)
    torch.cuda.synchronize()
    assert int(eng.status.cpu()[0]) == -1
    tl = c.tilt.reshape(-1, 2)[idx]
    L, _, _, _, r_tilt = P.grad_model_grads(
        c.geom(), c.probe, c.obj, c.scan.reshape(-1, 2)[idx], c.patterns.reshape(-1, *c.probe.shape[-2:])[idx],
        c.mask, c.props(), tl, onoise, with_tilt=True)
    assert float(loss.cpu()[0]) == pytest.approx(float(L), rel=1e-5)
    assert rel_l2(g_tilt.cpu().numpy()[idx], r_tilt) < 1e-3


def test_run_engine_with_tilt_updates_matches_oracle():
    c = make_case(seed=95, N=64, M=1, S=3, scan_shape=(4, 4))
    props = PL.GradientEnginePlan(
        solvers={'object': {'type': 'sgd', 'learning_rate': 2.0},
                 'tilt': {'type': 'adam', 'learning_rate': 0.5}},
        noise_model={'type': 'poisson', 'eps': 1e-3}, niter=3, grouping=8, update_tilt=True)
    state = run_engine({'data': Patterns(c.patterns, c.mask), 'state': make_state(c), 'dtype': numpy.float32,
                        'seed': 'tilt-seed', 'recons_name': 't'}, props)
    run = P.GradientRun(solvers={('object',): ('sgd', dict(learning_rate=2.0)),
                                 ('tilt',): ('adam', dict(learning_rate=0.5))},
                        niter=3, grouping=8, seed='tilt-seed', noise=P.NoiseModel(kind='poisson', eps=1e-3),
                        update_tilt=True)
    probe, obj, scan, losses, tilt = P.run_gradient(
        run, probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
        probe_sampling=c.probe_sampling, corner=c.osamp.corner, obj_sampling=c.osamp.sampling,
        thicknesses=c.thick, wavelength=c.wavelength, return_tilt=True)
    assert numpy.allclose(state.progress.detector_errors, losses, rtol=1e-4)
    assert rel_l2(state.object.data, obj) < 1e-4
    assert numpy.max(numpy.abs(state.tilt.reshape(-1, 2) - tilt)) < 1e-3 * max(1.0, numpy.max(numpy.abs(tilt)))
    assert numpy.max(numpy.abs(tilt)) > 0.1   # the tilts moved
