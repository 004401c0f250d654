"""The oracle's constraints and cost regularisers against the reference's own
outputs (tests/golden/constraints.npz, written by make_golden.py from
phaser/engines/common/regularizers.py), and the cost gradients against float64
central finite differences."""
import os

import numpy
import pytest

from oracle import phaser_np as P

from .conftest import GOLDEN


@pytest.fixture(scope='module')
def g():
    return dict(numpy.load(os.path.join(GOLDEN, 'constraints.npz'), allow_pickle=False))


def rel_l2(a, b):
    return float(numpy.linalg.norm(numpy.asarray(a, complex) - b) / numpy.linalg.norm(b))


def test_layers_matches_reference(g):
    out = P.regularize_layers(g['obj'], g['thick'], 30.0, 0.6)
    assert rel_l2(out, g['layers']) < 1e-6


def test_fourier_filters_match_reference(g):
    shape = g['obj'].shape[-2:]
    assert rel_l2(P.fourier_filter(g['obj'], P.low_pass_filter(shape, 0.3)), g['low_pass']) < 1e-6
    filt = P.gaussian_filter(shape, g['obj_sampling'], 0.7, 0.8)
    assert rel_l2(P.fourier_filter(g['obj'], filt), g['gaussian']) < 1e-6


def test_phase_ramp_matches_reference(g):
    rows, cols = P.region_crop(g['obj'].shape[-2:], g['corner'], g['obj_sampling'], g['region_min'],
                               g['region_max'])
    assert rel_l2(P.remove_phase_ramp(g['obj'], rows, cols), g['phase_ramp']) < 1e-6


def test_clamp_and_probe_support_fixtures_are_consistent(g):
    o = g['obj']
    m = numpy.abs(o)
    assert rel_l2(o * (numpy.minimum(m, numpy.float32(1.1)) / m), g['clamp']) < 1e-7
    N = g['probe'].shape[-1]
    ky, kx = P.recip_grid((N, N), g['probe_sampling'])
    mask = kx ** 2 + ky ** 2 <= (20.0 * 1e-3 / float(g['wavelength'])) ** 2
    assert rel_l2(P.ifft2c(P.fft2c(g['probe']) * mask), g['probe_support']) < 1e-6


COSTS = {'obj_l1': 0.3, 'obj_l2': 0.4, 'obj_phase_l1': 0.5, 'obj_tv': 0.6, 'obj_tikh': 0.7,
         'layers_tv': 0.8, 'layers_tikh': 0.9}


@pytest.mark.parametrize('name', list(COSTS))
def test_cost_values_match_reference(g, name):
    ref = dict(zip(g['cost_names'], g['cost_values']))[name]
    n_pos = g['scan'].shape[0] * g['scan'].shape[1]
    scale = float(g['cost_group_size']) / n_pos
    eps = 1e-6 if name == 'obj_tv' else 1e-8
    val, _ = P.obj_regularizer_costs(g['obj'], {name: COSTS[name]}, scale, tv_eps=eps)
    assert val == pytest.approx(ref, rel=2e-5)


@pytest.mark.parametrize('name', list(COSTS))
def test_cost_gradients_match_finite_differences(name):
    rng = numpy.random.default_rng(9)
    obj = (numpy.exp(1j * rng.normal(0, 0.6, (3, 9, 11))) * rng.uniform(0.7, 1.3, (3, 9, 11)))
    costs = {name: COSTS[name]}
    _, grad = P.obj_regularizer_costs(obj, costs, 0.25, tv_eps=1e-3)
    h = 1e-6
    for _ in range(24):
        s, y, x = rng.integers(3), rng.integers(9), rng.integers(11)
        for unit, part in ((1.0, grad.real), (1j, grad.imag)):
            op, om = obj.copy(), obj.copy()
            op[s, y, x] += h * unit
            om[s, y, x] -= h * unit
            fd = (P.obj_regularizer_costs(op, costs, 0.25, tv_eps=1e-3)[0]
                  - P.obj_regularizer_costs(om, costs, 0.25, tv_eps=1e-3)[0]) / (2 * h)
            assert fd == pytest.approx(part[s, y, x], rel=1e-4, abs=1e-6)


def test_fourier_and_probe_costs_match_reference(g):
    ref = dict(zip(g['cost_names'], g['cost_values']))
    n_pos = g['scan'].shape[0] * g['scan'].shape[1]
    scale = float(g['cost_group_size']) / n_pos
    v, _ = P.obj_recip_l1(g['obj'].astype(numpy.complex128), 0.01, scale)
    assert v == pytest.approx(ref['obj_recip_l1'], rel=1e-4)
    # the phase of fft2(P) outside the probe aperture is the phase of rounding noise, so
    # probe_phase_tikh depends on the FFT's rounding (complex64 here as in the reference):
    # its value agrees to a few percent only
    for name, cost, rel in (('probe_phase_tikh', 0.02, 3e-2), ('probe_recip_tikh', 0.03, 1e-4),
                            ('probe_recip_tv', 0.04, 1e-4)):
        v, _ = P.probe_regularizer_costs(g['probe'], {name: cost}, tv_eps=1e-8)
        assert v == pytest.approx(ref[name], rel=rel), name


def test_fourier_and_probe_cost_gradients_match_finite_differences():
    rng = numpy.random.default_rng(10)
    obj = numpy.exp(1j * rng.normal(0, 0.5, (2, 7, 9))) * rng.uniform(0.8, 1.2, (2, 7, 9))
    probe = (rng.normal(size=(2, 8, 8)) + 1j * rng.normal(size=(2, 8, 8)))
    h = 1e-6
    cases = [(lambda o: P.obj_recip_l1(o, 0.3, 0.5), obj)]
    for name in ('probe_phase_tikh', 'probe_recip_tikh', 'probe_recip_tv'):
        cases.append((lambda p, name=name: P.probe_regularizer_costs(p, {name: 0.7}, tv_eps=1e-3), probe))
    for f, x in cases:
        _, grad = f(x)
        for _ in range(10):
            i = tuple(rng.integers(s) for s in x.shape)
            for unit, part in ((1.0, grad.real), (1j, grad.imag)):
                xp, xm = x.copy(), x.copy()
                xp[i] += h * unit
                xm[i] -= h * unit
                fd = (f(xp)[0] - f(xm)[0]) / (2 * h)
                assert fd == pytest.approx(part[i], rel=1e-4, abs=1e-6)


def test_tilt_gaussian_matches_reference(g):
    out = P.unstructured_gaussian(g['tilt_in'].astype(numpy.float64), g['scan'], g['obj'].shape[-2:], g['corner'],
                                  g['obj_sampling'], 0.8, 0.7)
    assert numpy.max(numpy.abs(out - g['tilt_gaussian'])) < 1e-6 * numpy.max(numpy.abs(g['tilt_gaussian']))
