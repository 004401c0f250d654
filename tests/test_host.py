"""Host-side logic of the backend against the reference fixtures (CPU only)."""
import json
import os

import numpy
import pytest
from numpy.testing import assert_array_equal, assert_allclose

from phaser_b200 import groups as G
from phaser_b200 import plan as P
from phaser_b200 import optics
from phaser_b200.sampling import ObjectSampling, Sampling

from .conftest import GOLDEN


def load(name):
    return dict(numpy.load(os.path.join(GOLDEN, name), allow_pickle=False))


def test_groupings_bit_exact_with_reference():
    g = json.load(open(os.path.join(GOLDEN, 'groupings.json')))
    assert [a.tolist() for a in G.create_sparse_groupings(32, 8, 'seed1')] == g['sparse_32_8']
    assert [a.tolist() for a in G.create_sparse_groupings(33, 8, 'seed1')] == g['sparse_33_8']
    assert [a.tolist() for a in G.create_sparse_groupings((6, 7), 10, 'abc', i=3)] == g['sparse_6x7_10_i3']
    assert [int(v) for v in G.shuffled(list(range(5)), seed='abc', i=2)] == g['shuffle_5_i2']
    assert G.mask_fraction_of_groups(17, 0.1).tolist() == g['mask_17_0.1']
    assert G.mask_fraction_of_groups(3, 0.5).tolist() == g['mask_3_0.5']
    scan = numpy.stack(numpy.meshgrid(numpy.linspace(0., 20., 8), numpy.linspace(0., 20., 8),
                                      indexing='ij'), axis=-1).reshape(-1, 2)
    assert [a.tolist() for a in G.create_compact_groupings(scan, 16, 'seed1')] == g['compact_64_16']


def test_group_manager_iteration_semantics():
    gm = G.GroupManager((5, 6), 7, seed='s')
    first = gm.iter(None, 0)
    assert sum(g.shape[1] for g in first) == 30 and len(first) == len(gm) == 5
    again = gm.iter(None, 2, shuffle_groups=False)      # same groups, shuffled order
    assert sorted(map(lambda a: tuple(a.ravel()), again)) == sorted(map(lambda a: tuple(a.ravel()), first))
    fresh = gm.iter(None, 2, shuffle_groups=True)       # regenerated with entropy groupings_2
    assert [a.tolist() for a in fresh] == [a.tolist() for a in G.create_sparse_groupings((5, 6), 7, 's', 2)]
    flat = gm.flat(fresh[0])
    assert flat.dtype == numpy.int64 and flat.tolist() == (fresh[0][0] * 6 + fresh[0][1]).tolist()


def test_object_sampling_indices_bit_exact():
    g = load('cutouts.npz')
    osamp = ObjectSampling((60, 70), g['sampling'], g['corner'])
    shape = tuple(g['shape'])
    assert_array_equal(osamp.pos_to_object_idx(g['pos'], shape), g['idx'])
    assert_array_equal(osamp.cutout_starts(g['pos'], shape), g['starts'])
    assert_array_equal(osamp.get_subpx_shifts(g['pos'], shape), g['subpx'])


def test_propagators_match_reference():
    g = load('numerics.npz')
    samp = Sampling((32, 32), sampling=g['psamp'])
    ky, kx = samp.recip_grid(dtype=numpy.float32)
    props = optics.make_propagators(ky, kx, g['psamp'], float(g['wavelength']), g['thick'])
    assert_array_equal(props, g['props'])     # same float32 ops, same values
    probe = optics.make_focused_probe(ky, kx, float(g['wavelength']), 25., defocus=200.)
    assert numpy.linalg.norm(probe - g['probe']) / numpy.linalg.norm(g['probe']) < 1e-6
    modes = optics.make_hermite_modes(probe, 4, 0.7, [0.5, 1 / 3, 1 / 6])
    assert numpy.linalg.norm(modes - g['modes']) / numpy.linalg.norm(g['modes']) < 1e-5
    assert optics.electron_wavelength(200e3) == pytest.approx(0.02507934741, rel=1e-10)


def test_plan_hook_resolution():
    assert P.solver({'type': 'lsqml', 'beta_object': 0.5})[1].beta_object == 0.5
    assert P.solver('epie')[0] == 'epie'
    kind, props = P.noise_model({'type': 'anscombe'})
    assert kind == 'anscombe' and props.offset == 0.375
    assert P.position_solver({'type': 'momentum', 'step_size': 1e-3}) [1].momentum == 0.9

    class RefHook:   # the shape of phaser's Hook objects (phaser/hooks/hook.py:15-30)
        ref = 'phaser.engines.conventional.solvers:LSQMLSolver'
        type = 'lsqml'
        props = P.LSQMLSolverPlan(gamma=1e-3)
    assert P.solver(RefHook())[1].gamma == 1e-3
    with pytest.raises(NotImplementedError):
        P.solver('something_else')


def test_flags_and_schedules():
    class S:
        class iter:
            engine_iter = 6
    args = {'state': S, 'niter': 10}
    assert P.process_flag(True)(args) and not P.process_flag(False)(args)
    assert P.process_flag({'after': 5})(args)
    assert not P.process_flag(P.Flag(after=5, every=2))(args)
    assert not P.process_flag(P.Flag(before=6))(args)
    assert P.process_schedule(0.25)(args) == 0.25


def test_schedule_hooks_in_plan_form():
    """phaser/hooks/schedule.py:33-75: constant, piecewise (largest step <= i), expr."""
    class S:
        class iter:
            engine_iter = 6
    args = {'state': S, 'niter': 10}
    assert P.process_schedule({'type': 'constant', 'value': 3})(args) == 3.0
    pw = {'type': 'piecewise', 'init': 1.0, 'steps': {5: 0.5, 8: {'type': 'constant', 'value': 0.1}}}
    assert P.process_schedule(pw)(args) == 0.5
    S.iter.engine_iter = 9
    assert P.process_schedule(pw)(args) == pytest.approx(0.1)
    S.iter.engine_iter = 2
    assert P.process_schedule(pw)(args) == 1.0
    assert P.process_schedule({'type': 'expr', 'expr': '0.5 ** i / niter'})(args) == pytest.approx(0.025)
    with pytest.raises(NotImplementedError):
        P.process_schedule({'type': 'cosine'})


def test_defocus_and_propagation_signs_agree():
    """Known answer of the reference's test_propagator_sign (tests/test_optics.py:43-57),
    restated A against B instead of against its image fixture: a probe 200 A underfocused,
    propagated 200 A, is the focused probe; with either sign flipped it is not."""
    samp = Sampling((256, 256), extent=(25., 25.))
    ky, kx = samp.recip_grid(dtype=numpy.float32)

    def propagate(probe, dz):
        k = numpy.fft.fft2(numpy.fft.ifftshift(probe, axes=(-2, -1)), norm='ortho')
        k = k * optics.fresnel_propagator(ky, kx, 0.0251, dz)
        return numpy.fft.fftshift(numpy.fft.ifft2(k, norm='ortho'), axes=(-2, -1))

    focused = optics.make_focused_probe(ky, kx, 0.0251, 10., defocus=0.)
    under = optics.make_focused_probe(ky, kx, 0.0251, 10., defocus=-200.)
    scale = numpy.abs(focused).max()
    assert numpy.abs(numpy.abs(propagate(under, 200.)) - numpy.abs(focused)).max() < 1e-5 * scale
    assert numpy.abs(numpy.abs(propagate(under, -200.)) - numpy.abs(focused)).max() > 1e-2 * scale
    over = optics.make_focused_probe(ky, kx, 0.0251, 10., defocus=200.)
    assert numpy.abs(numpy.abs(propagate(over, 200.)) - numpy.abs(focused)).max() > 1e-2 * scale


def test_object_slicing_rounding():
    """Known answers of the reference's test_object_slicing (tests/test_object.py:105-143):
    an exact pixel position maps to that pixel, a shift under half a sample keeps it, and odd
    (2n + 1) and even (2n) cutouts n and n - 1/2 samples away start at the same pixel."""
    samp = ObjectSampling((40, 31), (0.5, 2.0))
    yy = samp.corner[0] + samp.sampling[0] * numpy.arange(40)
    xx = samp.corner[1] + samp.sampling[1] * numpy.arange(31)
    yp, xp = samp.cutout_starts(numpy.array((-1.25, 12.0)), (1, 1))
    assert yy[yp] == pytest.approx(-1.25) and xx[xp] == pytest.approx(12.0)
    assert_array_equal(samp.cutout_starts(numpy.array((-1.25 + 0.24, 12.0 - 0.99)), (1, 1)), (yp, xp))
    n = 2
    pos = numpy.array((-1.25 - 0.24 + 0.5 * n, 12.0 - 0.99 + 2.0 * n))
    assert_array_equal(samp.cutout_starts(pos, (2 * n + 1, 2 * n + 1)), (yp, xp))
    n = 6
    pos = numpy.array((-1.25 - 0.24 + 0.5 * (n - 0.5), 12.0 - 0.99 + 2.0 * (n - 0.5)))
    assert_array_equal(samp.cutout_starts(pos, (2 * n, 2 * n)), (yp, xp))
