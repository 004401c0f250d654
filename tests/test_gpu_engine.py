"""GPU parity of the fused multislice engine against the numpy oracle
(itself pinned to the reference by test_oracle_golden.py).

Tolerances (complex64 arithmetic, float64 step-size sums on the GPU, float32
sums in the oracle): forward model within 1e-5 relative L2; one mini-batch
step's object / probe within 1e-5 relative L2 of the oracle (their UPDATES
within 1e-3); per-position errors within 1e-4; position steps within 2e-3
(a ratio of two float32-accumulated sums in the oracle)."""
import numpy
import pytest
import torch

from oracle import phaser_np as P
from phaser_b200 import _lib
from phaser_b200.device import DeviceEngine, NoiseSpec
from phaser_b200.engines.conventional import run_engine
from phaser_b200 import plan as PL
from phaser_b200.state import ReconsState, ProbeState, ObjectState, IterState, Patterns
from phaser_b200.sampling import Sampling

from .cases import make_case

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = numpy.asarray(a, numpy.complex128)
    b = numpy.asarray(b, numpy.complex128)
    return float(numpy.linalg.norm(a - b) / numpy.linalg.norm(b))


def engine_for(c, group_max, noise=NoiseSpec()):
    return DeviceEngine(probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
                        probe_sampling=c.probe_sampling, obj_sampling=c.osamp, thicknesses=c.thick,
                        wavelength=c.wavelength, tilt=c.tilt, noise=noise, group_max=group_max)


CONFIGS = [
    dict(seed=1, N=64, M=1, S=1),
    dict(seed=2, N=64, M=2, S=3),
    dict(seed=3, N=128, M=4, S=2),
    dict(seed=4, N=64, M=3, S=2, tilt=True),
    dict(seed=5, N=128, M=1, S=3, scan_shape=(3, 3)),
    dict(seed=6, N=256, M=8, S=4, scan_shape=(2, 2)),
    dict(seed=7, N=256, M=2, S=3, scan_shape=(2, 2), tilt=True),
]


@pytest.mark.parametrize('cfg', CONFIGS, ids=lambda c: f"N{c['N']}M{c['M']}S{c['S']}{'t' if c.get('tilt') else ''}")
def test_forward_model_matches_oracle(cfg):
    c = make_case(**cfg)
    n = c.scan.shape[0] * c.scan.shape[1]
    eng = engine_for(c, n)
    idx = numpy.arange(n, dtype=numpy.int64)
    gt, sizes = eng.group_tensor([idx])
    sim = eng.simulate(gt[0], sizes[0]).cpu().numpy()
    g = c.geom()
    flat = c.scan.reshape(-1, 2)
    psi0, cuts, _, _ = P.cutout_group(g, c.probe, c.obj, flat)
    pt = P.tilt_propagators(g.ky, g.kx, c.thick, c.props(), None if c.tilt is None else c.tilt.reshape(-1, 2))
    psi = P._forward(psi0, cuts, pt)
    ref = numpy.sum(P.abs2(P.fft2c(psi[-1] * cuts[:, -1, None])), axis=1)
    assert rel_l2(sim, ref) < 1e-5


def run_group(c, solver, flags_kw, params, noise=P.NoiseModel()):
    n = c.scan.shape[0] * c.scan.shape[1]
    rng = numpy.random.default_rng(99)
    idx = rng.permutation(n)[: max(2, (2 * n) // 3)].astype(numpy.int64)
    spec = NoiseSpec('anscombe' if noise.offset else 'amplitude', noise.eps, noise.offset, noise.gaussian_variance)
    eng = engine_for(c, len(idx), spec)
    gt, sizes = eng.group_tensor([idx])
    flags = (_lib.PHB_FLAG_CALC_ERROR
             | (_lib.PHB_FLAG_UPDATE_OBJECT if flags_kw.get('update_object', True) else 0)
             | (_lib.PHB_FLAG_UPDATE_PROBE if flags_kw.get('update_probe', True) else 0)
             | (_lib.PHB_FLAG_UPDATE_POSITION if flags_kw.get('update_position', True) else 0))
    eng.status.fill_(-1)
    if solver == 'lsqml':
        eng.step('lsqml', gt[0], sizes[0], flags=flags, beta_object=params.beta_object,
                 beta_probe=params.beta_probe, illum_reg_object=params.illum_reg_object,
                 illum_reg_probe=params.illum_reg_probe, gamma=params.gamma)
    else:
        eng.step('epie', gt[0], sizes[0], flags=flags, beta_object=params.beta_object,
                 beta_probe=params.beta_probe)
    probe, obj, _ = eng.host_state()
    errors = eng.errors.cpu().numpy()[idx]
    pos = eng.pos_update.cpu().numpy()[idx]
    assert int(eng.status.cpu()[0]) == -1
    g = c.geom()
    tl = None if c.tilt is None else c.tilt.reshape(-1, 2)[idx]
    fn = P.lsqml_group if solver == 'lsqml' else P.epie_group
    ref = fn(g, c.probe, c.obj, c.scan.reshape(-1, 2)[idx], c.patterns.reshape(-1, *c.probe.shape[-2:])[idx],
             c.mask, c.props(), tl, noise, params, **flags_kw)
    return dict(obj=obj, probe=probe, errors=errors, pos=pos), ref


GROUP_CONFIGS = [
    ('lsqml', dict(seed=21, N=64, M=2, S=3), {}),
    ('lsqml', dict(seed=22, N=128, M=4, S=2), {}),
    ('lsqml', dict(seed=23, N=64, M=1, S=1), {}),
    ('lsqml', dict(seed=24, N=64, M=2, S=2, tilt=True), {}),
    ('lsqml', dict(seed=25, N=128, M=2, S=2), dict(update_probe=False)),
    ('epie', dict(seed=26, N=64, M=2, S=3), {}),
    ('epie', dict(seed=27, N=128, M=1, S=2), {}),
    ('lsqml', dict(seed=28, N=64, M=2, S=8, scan_shape=(3, 3)), {}),
    ('epie', dict(seed=29, N=64, M=1, S=6, scan_shape=(3, 3)), {}),
    ('lsqml', dict(seed=30, N=256, M=8, S=4, scan_shape=(3, 3)), {}),
    ('lsqml', dict(seed=32, N=256, M=2, S=2, scan_shape=(2, 2), tilt=True), {}),
]


@pytest.mark.parametrize('solver,cfg,flags', GROUP_CONFIGS,
                         ids=[f"{s}-N{c['N']}M{c['M']}S{c['S']}-{i}" for i, (s, c, f) in enumerate(GROUP_CONFIGS)])
def test_group_step_matches_oracle(solver, cfg, flags):
    c = make_case(**cfg)
    params = (P.LSQMLParams(0.9, 0.8, 1e-2, 1e-2, 1e-4) if solver == 'lsqml' else P.EPIEParams(0.7, 0.6))
    got, ref = run_group(c, solver, dict(flags, update_position=True), params)
    d_obj = rel_l2(got['obj'] - c.obj, ref['object'] - c.obj)
    d_probe = rel_l2(got['probe'] - c.probe, ref['probe'] - c.probe) if flags.get('update_probe', True) else 0.0
    assert rel_l2(got['obj'], ref['object']) < 1e-5, d_obj
    assert rel_l2(got['probe'], ref['probe']) < 1e-5, d_probe
    assert d_obj < 1e-3
    assert d_probe < 1e-3
    assert numpy.allclose(got['errors'], ref['errors'], rtol=1e-4)
    assert rel_l2(got['pos'], ref['pos_update']) < 2e-3


@pytest.mark.parametrize('solver,cfg', [('lsqml', dict(seed=21, N=64, M=2, S=3)), ('epie', dict(seed=26, N=64, M=2, S=3)),
                                        ('lsqml', dict(seed=22, N=128, M=4, S=2))])
def test_repeated_group_step_differs_by_reordering_noise_only(solver, cfg):
    """The float32 accumulators are summed with atomics, so two runs of the same step may
    differ in the order of their additions: the noise floor, 1e-6 here, is an order of
    magnitude under the 1e-5 parity tolerance, so a parity failure is not reordering."""
    c = make_case(**cfg)
    params = (P.LSQMLParams(0.9, 0.8, 1e-2, 1e-2, 1e-4) if solver == 'lsqml' else P.EPIEParams(0.7, 0.6))
    a, _ = run_group(c, solver, dict(update_position=True), params)
    b, _ = run_group(c, solver, dict(update_position=True), params)
    assert rel_l2(a['obj'], b['obj']) < 1e-6
    assert rel_l2(a['probe'], b['probe']) < 1e-6
    assert numpy.allclose(a['errors'], b['errors'], rtol=1e-5)


@pytest.mark.parametrize('N', [64, 256])
def test_presolve_rescale_matches_oracle(N):
    c = make_case(seed=31, N=N, M=2, S=3, scan_shape=(4, 4) if N == 64 else (3, 3))
    n = c.scan.shape[0] * c.scan.shape[1]
    eng = engine_for(c, 8)
    flat = numpy.arange(n, dtype=numpy.int64)
    chunks = [flat[i:i + 8] for i in range(0, n, 8)]
    gt, sizes = eng.group_tensor(chunks)
    r = eng.presolve(gt, sizes, 'lsqml')
    g = c.geom()
    ref = []
    for ch in chunks:
        ref.append(P.epie_dry_run(g, c.probe, c.obj, c.scan.reshape(-1, 2)[ch],
                                  c.patterns.reshape(-1, N, N)[ch], c.mask, c.props(), None))
    assert r == pytest.approx(float(numpy.mean(numpy.concatenate(ref))), rel=1e-5)


def make_state(c):
    N = c.probe.shape[-1]
    return ReconsState(iter=IterState(), wavelength=c.wavelength,
                       probe=ProbeState(Sampling((N, N), sampling=c.probe_sampling), c.probe.copy()),
                       object=ObjectState(c.osamp, c.obj.copy(), c.thick.copy()),
                       scan=c.scan.copy(), tilt=None)


@pytest.mark.parametrize('solver', ['lsqml', 'epie'])
def test_run_engine_matches_oracle(solver):
    c = make_case(seed=41, N=64, M=2, S=2, scan_shape=(5, 5))
    props = PL.ConventionalEnginePlan(
        noise_model={'type': 'amplitude', 'eps': 1e-2},
        solver=({'type': 'lsqml', 'beta_object': 0.9, 'beta_probe': 0.8, 'gamma': 1e-3} if solver == 'lsqml'
                else {'type': 'epie', 'beta_object': 0.9, 'beta_probe': 0.8}),
        position_solver={'type': 'momentum', 'step_size': 1e-2, 'max_step_size': 0.2, 'momentum': 0.9},
        niter=3, grouping=10, update_positions=True, calc_error_fraction=0.5)
    state = run_engine({'data': Patterns(c.patterns, c.mask), 'state': make_state(c), 'dtype': numpy.float32,
                        'seed': 'engine-seed', 'recons_name': 't'}, props)
    run = P.ConventionalRun(solver=solver, niter=3, grouping=10, seed='engine-seed', noise=P.NoiseModel(eps=1e-2),
                            lsqml=P.LSQMLParams(0.9, 0.8, 1e-2, 1e-2, 1e-3), epie=P.EPIEParams(0.9, 0.8),
                            update_positions=True, position_solver='momentum', pos_step_size=1e-2,
                            pos_max_step=0.2, pos_momentum=0.9, calc_error_fraction=0.5)
    probe, obj, scan, errors = P.run_conventional(
        run, probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
        probe_sampling=c.probe_sampling, corner=c.osamp.corner, obj_sampling=c.osamp.sampling,
        thicknesses=c.thick, wavelength=c.wavelength)
    assert rel_l2(state.object.data, obj) < 1e-4
    assert rel_l2(state.probe.data, probe) < 1e-4
    assert numpy.max(numpy.abs(state.scan - scan)) < 1e-4
    assert numpy.allclose(state.progress.detector_errors, errors, rtol=1e-3)


def test_run_engine_matches_oracle_n256():
    """Two whole LSQ-ML iterations at a 256^2 probe and detector (4-CTA cluster tiles): sparse
    shuffled groups, presolve, momentum position correction, per-iteration errors."""
    c = make_case(seed=43, N=256, M=4, S=2, scan_shape=(3, 3))
    props = PL.ConventionalEnginePlan(
        noise_model={'type': 'amplitude', 'eps': 1e-2},
        solver={'type': 'lsqml', 'beta_object': 0.9, 'beta_probe': 0.8, 'gamma': 1e-3},
        position_solver={'type': 'momentum', 'step_size': 10.0, 'max_step_size': 0.2, 'momentum': 0.9},
        niter=2, grouping=5, update_positions=True, calc_error_fraction=1.0)
    state = run_engine({'data': Patterns(c.patterns, c.mask), 'state': make_state(c), 'dtype': numpy.float32,
                        'seed': 'engine-seed-256', 'recons_name': 't'}, props)
    run = P.ConventionalRun(solver='lsqml', niter=2, grouping=5, seed='engine-seed-256', noise=P.NoiseModel(eps=1e-2),
                            lsqml=P.LSQMLParams(0.9, 0.8, 1e-2, 1e-2, 1e-3), update_positions=True,
                            position_solver='momentum', pos_step_size=10.0, pos_max_step=0.2, pos_momentum=0.9,
                            calc_error_fraction=1.0)
    probe, obj, scan, errors = P.run_conventional(
        run, probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
        probe_sampling=c.probe_sampling, corner=c.osamp.corner, obj_sampling=c.osamp.sampling,
        thicknesses=c.thick, wavelength=c.wavelength)
    assert rel_l2(state.object.data, obj) < 1e-4
    assert rel_l2(state.probe.data, probe) < 1e-4
    # the positions move by ~3.5e-3 A over the two iterations: agree to ~3% of that
    assert numpy.max(numpy.abs(scan - c.scan)) > 1e-3
    assert numpy.max(numpy.abs(state.scan - scan)) < 1e-4
    assert numpy.allclose(state.progress.detector_errors, errors, rtol=1e-3)


def test_positions_leaving_the_object_raise_value_error():
    """An unclipped position step that throws the probe off the object ends the run with
    the reference's error (utils/object.py:288-289), counted on the device."""
    c = make_case(seed=44, N=64, M=1, S=1, scan_shape=(4, 4))
    props = PL.ConventionalEnginePlan(
        noise_model={'type': 'amplitude'}, solver={'type': 'lsqml'},
        position_solver={'type': 'momentum', 'step_size': 1e9, 'max_step_size': None, 'momentum': 0.0},
        niter=2, grouping=8, update_positions=True)
    with pytest.raises(ValueError, match='probe positions completely outside object'):
        run_engine({'data': Patterns(c.patterns, c.mask), 'state': make_state(c), 'dtype': numpy.float32,
                    'seed': 'outside', 'recons_name': 't'}, props)


def test_nonfinite_pattern_raises_value_error():
    c = make_case(seed=51, N=64, M=1, S=1, scan_shape=(4, 4))
    c.patterns[1, 2, 5, 5] = numpy.inf
    props = PL.ConventionalEnginePlan(niter=1, grouping=8)
    with pytest.raises(ValueError, match="NaN or inf encountered in object or probe, group"):
        run_engine({'data': Patterns(c.patterns, c.mask), 'state': make_state(c), 'dtype': numpy.float32,
                    'seed': 1, 'recons_name': 't'}, props)


def test_unsupported_shapes_fail_loudly():
    c = make_case(seed=52, N=64, M=1, S=1, scan_shape=(2, 2))
    with pytest.raises(NotImplementedError):
        DeviceEngine(probe=numpy.zeros((1, 96, 96), numpy.complex64), obj=c.obj, scan=c.scan,
                     patterns=numpy.zeros((4, 96, 96), numpy.float32), mask=numpy.ones((96, 96), numpy.float32),
                     probe_sampling=c.probe_sampling, obj_sampling=c.osamp, thicknesses=c.thick,
                     wavelength=c.wavelength)
    eng = engine_for(c, 2)
    with pytest.raises(ValueError):
        eng.group_tensor([numpy.arange(4)])
    # ePIE needs every mode of a position in one cluster: not at a 256 x 256 probe
    c2 = make_case(seed=53, N=256, M=2, S=2, scan_shape=(2, 2))
    eng = engine_for(c2, 4)
    gt, sizes = eng.group_tensor([numpy.arange(4)])
    with pytest.raises(NotImplementedError):
        eng.step('epie', gt[0], sizes[0], flags=_lib.PHB_FLAG_UPDATE_OBJECT)


@pytest.mark.parametrize('solver,N', [('lsqml', 64), ('epie', 64), ('grad', 64), ('lsqml', 256), ('grad', 256)])
def test_uint16_resident_patterns_match_float32(solver, N):
    """Patterns held as uint16 counts give the float32 results (the kernels convert
    each count exactly): presolve rescale, one group step, errors / loss."""
    c = make_case(seed=55, N=N, M=2, S=3) if N == 64 else make_case(seed=56, N=N, M=2, S=2, scan_shape=(3, 3))
    n = c.scan.shape[0] * c.scan.shape[1]
    counts = numpy.round(c.patterns * (4000.0 / c.patterns.max())).astype(numpy.uint16)
    idx = numpy.random.default_rng(3).permutation(n)[:min(10, n)].astype(numpy.int64)
    spec = NoiseSpec('poisson', 1e-3, 0.0, 0.1) if solver == 'grad' else NoiseSpec()
    out = []
    for pats in (counts, counts.astype(numpy.float32)):
        eng = DeviceEngine(probe=c.probe, obj=c.obj, scan=c.scan, patterns=pats, mask=c.mask,
                           probe_sampling=c.probe_sampling, obj_sampling=c.osamp, thicknesses=c.thick,
                           wavelength=c.wavelength, noise=spec, group_max=len(idx))
        assert eng.patterns.dtype == (torch.uint16 if pats.dtype == numpy.uint16 else torch.float32)
        gt, sizes = eng.group_tensor([idx])
        rescale = eng.presolve(gt, sizes, 'epie' if solver == 'epie' else 'lsqml', gradient_form=solver == 'grad')
        flags = (_lib.PHB_FLAG_UPDATE_OBJECT | _lib.PHB_FLAG_UPDATE_PROBE | _lib.PHB_FLAG_UPDATE_POSITION
                 | _lib.PHB_FLAG_CALC_ERROR)
        eng.status.fill_(-1)
        if solver == 'grad':
            g_obj, loss = torch.zeros_like(eng.object), torch.zeros((1,), dtype=torch.float64, device='cuda')
            eng.step('grad', gt[0], sizes[0], flags=_lib.PHB_FLAG_UPDATE_OBJECT, grad_object=g_obj, group_loss=loss)
            res = (rescale, g_obj.cpu().numpy(), float(loss.cpu()[0]))
        else:
            eng.step(solver, gt[0], sizes[0], flags=flags, beta_object=0.9, beta_probe=0.8)
            p, o, _ = eng.host_state()
            res = (rescale, o, p, eng.errors.cpu().numpy()[idx])
        assert int(eng.status.cpu()[0]) == -1
        out.append(res)
    (a, b) = out
    assert a[0] == pytest.approx(b[0], rel=1e-6)
    for x, y in zip(a[1:], b[1:]):
        if isinstance(x, float):
            assert x == pytest.approx(y, rel=1e-6)
        else:
            assert rel_l2(x, y) < 1e-6
