"""State preparation on the device (phaser_b200.prepare, csrc/phb_prepare.cu)
against the numpy oracle (oracle/prepare_np.py) and against the reference's own
prepare_for_engine outputs (tests/golden/prepare.npz): probe / pattern / mask
resizing (pad_crop and resample, up and down), object resampling and padding,
probe-mode truncation and creation, z reslicing.  Tolerance 1e-5 relative L2
(float32 interpolation against scipy's float64); grids exact."""
import numpy
import pytest
import torch

from oracle import prepare_np as PR
from phaser_b200 import prepare as DP
from phaser_b200.plan import ConventionalEnginePlan, SliceList, SliceStep, SliceTotal
from phaser_b200.sampling import ObjectSampling, Sampling
from phaser_b200.state import IterState, ObjectState, Patterns, ProbeState, ReconsState

from .test_gpu_engine import rel_l2
from .test_oracle_golden import load

pytestmark = pytest.mark.gpu

PLANS = {
    'pad_crop_up': dict(sim_shape=(40, 40), resize_method='pad_crop', probe_modes=2),
    'pad_crop_down': dict(sim_shape=(24, 24), resize_method='pad_crop', probe_modes=2),
    'resample_up': dict(sim_shape=(36, 36), resize_method='resample', probe_modes=2),
    'resample_down': dict(sim_shape=(28, 28), resize_method='resample', probe_modes=2, obj_pad_px=9.0),
    'modes_down': dict(probe_modes=1),
    'modes_up': dict(probe_modes=4, base_mode_power=0.6),
    'reslice': dict(probe_modes=2, slices=SliceStep(n=5, slice_thickness=10.0)),
    'reslice_total': dict(probe_modes=2, slices=SliceTotal(n=2, total_thickness=40.0)),
    'to_single': dict(probe_modes=2, slices=SliceList(thicknesses=[])),
}


@pytest.mark.parametrize('dtype', ['c64', 'f32'])
@pytest.mark.parametrize('recip', [False, True])
@pytest.mark.parametrize('shape,out,matrix,offset', [((19, 21), (20, 25), (1.0, 1.0), (-3.0, 2.0)),
                                                      ((32, 32), (40, 40), (0.8, 0.8), (3.1, 3.1)),
                                                      ((33, 30), (23, 17), (1.6, 0.7), (-4.5, 3.25))])
def test_resample_kernel_matches_oracle(dtype, recip, shape, out, matrix, offset):
    rng = numpy.random.default_rng(sum(shape) + recip)
    a = rng.normal(size=(3, *shape))
    if dtype == 'c64':
        a = (a + 1j * rng.normal(size=(3, *shape))).astype(numpy.complex64)
        cval = 0.5 - 0.25j
    else:
        a = a.astype(numpy.float32)
        cval = 0.75
    if recip:
        cval = 0.0
        ref = numpy.fft.ifftshift(PR.affine_linear(numpy.fft.fftshift(a, axes=(-1, -2)), matrix, offset, out, cval),
                                  axes=(-1, -2))
    else:
        ref = PR.affine_linear(a, matrix, offset, out, cval)
    got = DP._resample(torch.from_numpy(a).cuda(), out, matrix, offset, cval, recip)
    assert rel_l2(got.cpu().numpy(), ref) < 1e-6


@pytest.mark.parametrize('align', ['top', 'middle', 'bottom'])
@pytest.mark.parametrize('pad', ['vacuum', 'edge', 'average'])
def test_reslice_kernel_matches_reference(align, pad):
    g = load('prepare.npz')
    obj = g['object'][:, 20:32, 24:36]
    got = DP.resample_slices(torch.from_numpy(numpy.ascontiguousarray(obj)).cuda(), g['thicknesses'],
                             [12.0, 9.0, 14.0, 11.0], align=align, pad_mode=pad)
    assert rel_l2(got.cpu().numpy(), g[f'slices_{align}_{pad}']) < 1e-5


@pytest.mark.parametrize('old,new', [([], [8.0, 12.0, 20.0]), ([10.0, 10.0, 10.0], []), ([], []),
                                     ([5.0, 15.0], [7.0, 7.0, 6.0, 10.0])])
def test_reslice_special_cases_match_oracle(old, new):
    rng = numpy.random.default_rng(len(old) * 10 + len(new))
    S = max(1, len(old))
    obj = (numpy.exp(1j * rng.normal(0, 0.4, (S, 9, 11))) * rng.uniform(0.8, 1.0, (S, 9, 11))).astype(numpy.complex64)
    got = DP.resample_slices(torch.from_numpy(obj).cuda(), old, new).cpu().numpy()
    ref = PR.resample_slices(obj, old, new)
    assert got.shape == ref.shape and rel_l2(got, ref) < 1e-5


def golden_state(g):
    psamp = Sampling(g['probe'].shape[-2:], sampling=tuple(g['probe_sampling']))
    osamp = ObjectSampling(tuple(g['osamp_shape']), g['obj_sampling'], g['corner'], g['region_min'], g['region_max'])
    return ReconsState(iter=IterState(), wavelength=float(g['wavelength']), probe=ProbeState(psamp, g['probe'].copy()),
                       object=ObjectState(osamp, g['object'].copy(), g['thicknesses'].copy()), scan=g['scan'].copy())


@pytest.mark.parametrize('name', list(PLANS))
def test_prepare_for_engine_matches_reference(name):
    g = load('prepare.npz')
    pats, st = DP.prepare_for_engine(Patterns(g['patterns'].copy(), g['mask'].copy()), golden_state(g),
                                     ConventionalEnginePlan(**PLANS[name]))
    p = name + '__'
    os2 = st.object.sampling
    assert numpy.allclose(st.probe.sampling.sampling, g[p + 'probe_sampling'], rtol=1e-12)
    assert numpy.array_equal(os2.shape, g[p + 'obj_shape'])
    assert numpy.allclose(os2.sampling, g[p + 'obj_sampling'], rtol=1e-12)
    assert numpy.allclose(os2.corner, g[p + 'corner'], rtol=1e-12, atol=1e-12)
    assert numpy.allclose(os2.region_min, g[p + 'region_min']) and numpy.allclose(os2.region_max, g[p + 'region_max'])
    assert numpy.allclose(st.object.thicknesses, g[p + 'thicknesses'])
    assert torch.is_tensor(st.probe.data) and st.probe.data.is_cuda and torch.is_tensor(pats.patterns)
    ref_probe = g[p + 'probe']
    assert tuple(st.probe.data.shape) == ref_probe.shape and rel_l2(st.probe.data.cpu().numpy(), ref_probe) < 1e-5
    ref_obj = g[p + 'object'] if (p + 'object') in g else g['object']
    assert tuple(st.object.data.shape) == ref_obj.shape and rel_l2(st.object.data.cpu().numpy(), ref_obj) < 1e-5
    ref_pats = g[p + 'patterns'] if (p + 'patterns') in g else g['patterns']
    assert tuple(pats.patterns.shape) == ref_pats.shape and rel_l2(pats.patterns.cpu().numpy(), ref_pats) < 1e-5
    ref_mask = g[p + 'mask'] if (p + 'mask') in g else g['mask']
    assert rel_l2(pats.pattern_mask.cpu().numpy(), ref_mask) < 1e-5


def test_engine_runs_on_the_prepared_device_state():
    """64^2 probe resized to 128^2 (pad_crop) and reconstructed straight from the
    device tensors: the same result as the engine fed host copies of those arrays
    (within float32 atomic-order noise)."""
    from phaser_b200.engines.conventional import ConventionalEngine
    from phaser_b200.synthetic import epie_single_slice_config, simulate_patterns
    ds = epie_single_slice_config(seed=5)
    pats = simulate_patterns(ds, seed=5, device='cuda', group=64)
    N = ds.probe.shape[-1]

    def state():
        return ReconsState(iter=IterState(), wavelength=ds.wavelength,
                           probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling), ds.probe.copy()),
                           object=ObjectState(ds.obj_sampling, ds.init_object.copy(), ds.thicknesses.copy()),
                           scan=ds.scan.copy())

    plan = ConventionalEnginePlan(noise_model={'type': 'amplitude'}, solver={'type': 'lsqml'}, niter=2, grouping=64,
                                  sim_shape=(128, 128), resize_method='pad_crop', probe_modes=2)
    p_dev, st_dev = DP.prepare_for_engine(Patterns(pats, ds.mask), state(), plan)
    assert tuple(st_dev.probe.data.shape) == (2, 128, 128) and tuple(p_dev.patterns.shape[-2:]) == (128, 128)
    host = ReconsState(iter=IterState(), wavelength=ds.wavelength,
                       probe=ProbeState(st_dev.probe.sampling, st_dev.probe.data.cpu().numpy()),
                       object=ObjectState(st_dev.object.sampling, st_dev.object.data.cpu().numpy(),
                                          numpy.asarray(st_dev.object.thicknesses)),
                       scan=ds.scan.copy())
    results = []
    for data, st in ((p_dev, st_dev), (Patterns(p_dev.patterns.cpu().numpy(), p_dev.pattern_mask.cpu().numpy()), host)):
        eng = ConventionalEngine({'data': data, 'state': st, 'dtype': numpy.float32, 'seed': 'prep',
                                  'recons_name': 'prep'}, plan)
        eng.presolve()
        for i in (1, 2):
            eng.iteration(i)
        out = eng.finish()
        results.append((out.object.data.copy(), out.probe.data.copy()))
    assert rel_l2(results[0][0], results[1][0]) < 1e-5 and rel_l2(results[0][1], results[1][1]) < 1e-5
    assert numpy.all(numpy.isfinite(results[0][0]))


def test_take_state_continues_another_engines_reconstruction():
    """The gradient engine's result handed to LSQ-ML on the device equals starting
    LSQ-ML from host copies of that result."""
    from phaser_b200.engines.conventional import ConventionalEngine
    from phaser_b200.engines.gradient import GradientEngine
    from phaser_b200.plan import GradientEnginePlan
    from phaser_b200.synthetic import epie_single_slice_config, simulate_patterns
    ds = epie_single_slice_config(seed=6)
    pats = simulate_patterns(ds, seed=6, device='cuda', group=64)
    N = ds.probe.shape[-1]

    def state(probe=None, obj=None):
        return ReconsState(iter=IterState(), wavelength=ds.wavelength,
                           probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling),
                                            ds.probe.copy() if probe is None else probe),
                           object=ObjectState(ds.obj_sampling, ds.init_object.copy() if obj is None else obj,
                                              ds.thicknesses.copy()),
                           scan=ds.scan.copy())

    args = dict(dtype=numpy.float32, seed='handoff', recons_name='h')
    g = GradientEngine(dict(args, data=Patterns(None, ds.mask), state=state()),
                       # Anscombe: with one mode and a flat start some far-field intensities are exactly
                       # zero, where the amplitude model's d sqrt(I)/dI (jax's too) is infinite
                       GradientEnginePlan(solvers={'object': {'type': 'adam', 'learning_rate': 1e-2}},
                                          noise_model={'type': 'anscombe'}, niter=2, grouping=64),
                       patterns_on_device=pats)
    g.presolve()
    g.iteration(1)
    g.iteration(2)
    plan = ConventionalEnginePlan(noise_model={'type': 'amplitude'}, solver={'type': 'lsqml'}, niter=1, grouping=64)
    a = ConventionalEngine(dict(args, data=Patterns(None, ds.mask), state=state()), plan, patterns_on_device=pats)
    a.presolve()
    a.eng.take_state(g.eng)
    b = ConventionalEngine(dict(args, data=Patterns(None, ds.mask),
                                state=state(g.eng.probe.cpu().numpy(), g.eng.object.cpu().numpy())), plan,
                           patterns_on_device=pats)
    b.eng.take_state(g.eng)     # same probe scale: skip b's own presolve
    for e in (a, b):
        e.iteration(1)
    assert rel_l2(a.eng.object.cpu().numpy(), b.eng.object.cpu().numpy()) < 1e-5
    assert rel_l2(a.eng.probe.cpu().numpy(), b.eng.probe.cpu().numpy()) < 1e-5
    two_modes = numpy.concatenate([ds.probe, 0.1 * ds.probe]).astype(numpy.complex64)
    other = ConventionalEngine(dict(args, data=Patterns(None, ds.mask), state=state(probe=two_modes)), plan,
                               patterns_on_device=pats)
    with pytest.raises(ValueError):
        other.eng.take_state(g.eng)
