"""Pin the numpy oracle against fixtures produced by the reference itself
(tests/golden/make_golden.py).  CPU only."""
import json
import os

import numpy
import pytest
from numpy.testing import assert_allclose, assert_array_equal

from oracle import phaser_np as P

from .conftest import GOLDEN


def load(name):
    return dict(numpy.load(os.path.join(GOLDEN, name), allow_pickle=False))


def rel_l2(a, b):
    a = numpy.asarray(a, numpy.complex128)
    b = numpy.asarray(b, numpy.complex128)
    return float(numpy.linalg.norm(a - b) / max(numpy.linalg.norm(b), 1e-300))


# ---------------------------------------------------------------- numerics

def test_fft_conventions_match_reference():
    g = load('numerics.npz')
    for k in ('a8', 'a5'):
        assert rel_l2(P.fft2c(g[k]), g['fft_' + k]) < 1e-6
        assert rel_l2(P.ifft2c(g[k]), g['ifft_' + k]) < 1e-6


def test_fft_known_answers():
    # centred delta <-> constant, ortho normalisation (reference tests/test_num.py:102-155)
    a = numpy.pad(numpy.array([[5.]], numpy.float32), ((2, 2), (2, 2)))
    assert_allclose(P.fft2c(a), numpy.full((5, 5), 1., numpy.complex64), atol=1e-6)
    b = numpy.full((5, 5), 1 + 1j, numpy.complex64)
    assert_allclose(P.fft2c(b), numpy.pad([[5 + 5j]], ((0, 4), (0, 4))), atol=1e-5)
    c = numpy.pad(numpy.array([[5.]], numpy.float32), ((0, 4), (0, 4)))
    assert_allclose(P.ifft2c(c), numpy.full((5, 5), 1., numpy.complex64), atol=1e-5)
    assert_allclose(P.ifft2c(b), numpy.pad([[5 + 5j]], ((2, 2), (2, 2))), atol=1e-5)


def test_optics_match_reference():
    g = load('numerics.npz')
    ky, kx = P.recip_grid((32, 32), g['psamp'], numpy.float32)
    lam = float(g['wavelength'])
    probe = P.make_focused_probe(ky, kx, lam, 25., defocus=200.)
    assert rel_l2(probe, g['probe']) < 1e-6
    modes = P.hermite_modes(probe, 4, 0.7, [0.5, 1 / 3, 1 / 6])
    assert rel_l2(modes, g['modes']) < 1e-5
    assert rel_l2(P.fresnel_propagator(ky, kx, lam, 20., tilt=(3., -2.)), g['prop']) < 1e-6
    assert rel_l2(P.fourier_shift_filter(ky, kx, g['shifts']), g['filt']) < 1e-6
    props = P.make_propagators(ky, kx, g['psamp'], lam, g['thick'], 2 / 3)
    assert rel_l2(props, g['props']) < 1e-6
    assert_allclose(P.raster_scan((4, 5), (1.5, 2.0), numpy.float32), g['raster'])


def test_noise_losses_match_reference():
    g = load('noise_losses.npz')
    models = [P.NoiseModel(), P.NoiseModel.anscombe(), P.NoiseModel(kind='poisson')]
    for nm, ref in zip(models, g['losses']):
        assert float(nm.loss(g['intensity'], g['patterns'], g['mask'])) == pytest.approx(ref, rel=1e-5)


def test_groupings_and_constants_match_reference():
    g = json.load(open(os.path.join(GOLDEN, 'groupings.json')))
    assert [a.tolist() for a in P.sparse_groupings((32,), 8, 'seed1')] == g['sparse_32_8']
    assert [a.tolist() for a in P.sparse_groupings((33,), 8, 'seed1')] == g['sparse_33_8']
    assert [a.tolist() for a in P.sparse_groupings((6, 7), 10, 'abc', 3)] == g['sparse_6x7_10_i3']
    assert P.shuffled_order(5, 'abc', 2).tolist() == g['shuffle_5_i2']
    assert P.mask_fraction_of_groups(17, 0.1).tolist() == g['mask_17_0.1']
    assert P.mask_fraction_of_groups(3, 0.5).tolist() == g['mask_3_0.5']
    assert P.electron_wavelength(200e3) == pytest.approx(g['wavelength_200kV'], rel=1e-12)
    assert P.electron_wavelength(200e3) == pytest.approx(0.02507934741, rel=1e-10)


# ---------------------------------------------------------------- cutouts

def test_cutout_indices_bit_exact():
    g = load('cutouts.npz')
    shape = tuple(g['shape'])
    idx = P.object_index(g['pos'], g['corner'], g['sampling'], shape)
    assert_array_equal(idx, g['idx'])           # float64 bit-exact
    starts = P.cutout_starts(g['pos'], g['corner'], g['sampling'], shape)
    assert_array_equal(starts, g['starts'])     # integer bit-exact (round half even)
    assert_array_equal(P.subpx_shifts(g['pos'], g['corner'], g['sampling'], shape), g['subpx'])


def test_cutout_get_add_match_reference():
    g = load('cutouts.npz')
    shape = tuple(g['shape'])
    assert_array_equal(P.get_cutouts(g['obj'], g['starts'], shape), g['gathered'])
    added = P.add_cutouts(g['obj'].copy(), g['starts'], g['views'])
    assert_allclose(added, g['added'], rtol=0, atol=2e-6)


# ---------------------------------------------------------------- group steps

def group_inputs(g):
    N = g['probe'].shape[-1]
    rdt = P.real_dtype(g['probe'].dtype)
    ky, kx = P.recip_grid((N, N), g['probe_sampling'], rdt)
    geom = P.Geometry(g['corner'], g['obj_sampling'], ky, kx, g['thicknesses'])
    props = P.make_propagators(ky, kx, g['probe_sampling'], float(g['wavelength']), g['thicknesses'])
    scan = g['scan'].reshape(-1, 2)
    pats = g['patterns'].reshape(-1, N, N)
    idx = g['group']
    tilt = None if g['tilt'].size == 0 else g['tilt'].reshape(-1, 2)[idx]
    return geom, props, scan[idx], pats[idx], tilt


GROUP_CASES = ['lsqml_ms', 'lsqml_ss', 'lsqml_tilt', 'lsqml_noprobe', 'lsqml_f64', 'epie_ms', 'epie_ss']


@pytest.mark.parametrize('case', GROUP_CASES)
def test_group_step_matches_reference(case):
    g = load(f'group_{case}.npz')
    geom, props, gscan, gpats, tilt = group_inputs(g)
    noise = P.NoiseModel.anscombe() if str(g['noise']) == 'anscombe' else P.NoiseModel()
    uo, up = (bool(v) for v in g['flags'])
    f64 = g['probe'].dtype == numpy.complex128
    tol = 1e-10 if f64 else 2e-5
    if case.startswith('lsqml'):
        bo, bp, ro, rp, gm = g['params']
        prm = P.LSQMLParams(bo, bp, ro, rp, gm)
        res = P.lsqml_group(geom, g['probe'], g['object'], gscan, gpats, g['mask'], props, tilt,
                            noise, prm, update_object=uo, update_probe=up)
        om, pm, resc = P.lsqml_dry_run(geom, g['probe'], g['object'], gscan, gpats, g['mask'], props, tilt,
                                       numpy.zeros_like(g['dry_obj_mag']), numpy.zeros_like(g['dry_probe_mag']))
        assert rel_l2(om, g['dry_obj_mag']) < tol
        assert rel_l2(pm, g['dry_probe_mag']) < tol
        assert rel_l2(res['probe_mag'], g['new_probe_mag']) < tol
        assert rel_l2(res['obj_mag'], g['new_obj_mag']) < tol
    else:
        bo, bp = g['params']
        res = P.epie_group(geom, g['probe'], g['object'], gscan, gpats, g['mask'], props, tilt,
                           noise, P.EPIEParams(bo, bp), update_object=uo, update_probe=up)
        resc = P.epie_dry_run(geom, g['probe'], g['object'], gscan, gpats, g['mask'], props, tilt)
    assert rel_l2(resc, g['dry_rescale']) < tol
    assert rel_l2(res['object'], g['out_object']) < tol
    assert rel_l2(res['probe'], g['out_probe']) < tol
    assert rel_l2(res['errors'], g['errors']) < tol
    assert rel_l2(res['pos_update'], g['pos_update']) < (1e-9 if f64 else 1e-4)


@pytest.mark.parametrize('solver', ['lsqml', 'epie'])
def test_engine_run_matches_reference(solver):
    g = load(f'engine_{solver}.npz')
    run = P.ConventionalRun(solver=solver, niter=int(g['niter']), grouping=int(g['grouping']),
                            seed='golden-seed', noise=P.NoiseModel(eps=1e-2),
                            lsqml=P.LSQMLParams(0.9, 0.9, 1e-2, 1e-2, 1e-3), epie=P.EPIEParams(0.8, 0.7),
                            update_positions=True, position_solver='momentum', pos_step_size=1e-2,
                            pos_max_step=0.2, pos_momentum=0.9, calc_error_fraction=0.5)
    probe, obj, scan, errors = P.run_conventional(
        run, probe=g['probe'], obj=g['object'], scan=g['scan'], patterns=g['patterns'], mask=g['mask'],
        probe_sampling=g['probe_sampling'], corner=g['corner'], obj_sampling=g['obj_sampling'],
        thicknesses=g['thicknesses'], wavelength=float(g['wavelength']))
    assert rel_l2(obj, g['out_object']) < 1e-5
    assert rel_l2(probe, g['out_probe']) < 1e-5
    assert_allclose(scan, g['out_scan'], rtol=0, atol=1e-6)
    assert_allclose(errors, g['errors'], rtol=1e-5)


def test_cutout_multidim_known_answers():
    """Known answers of the reference's test_cutout_multidim (tests/test_object.py:265-295):
    a 2 x 2 grid of (80, 100) cutouts from a 3 x 200^2 ramp object, corner of the default
    centred grid, top-left values and unit ramps along x, 2 along y."""
    sampling = numpy.array([1.0, 1.0])
    corner = -numpy.array([200., 200.]) * sampling / 2. + sampling / 2.
    zz, yy, xx = numpy.indices((3, 200, 200), dtype=numpy.float32)
    obj = 1000. * zz + (2. * yy + xx)
    pos = numpy.array([[[-50., -50.], [-50., 50.]], [[50., -50.], [50., 50.]]])
    starts = P.cutout_starts(pos.reshape(-1, 2), corner, sampling, (80, 100))
    cut = P.get_cutouts(obj, starts, (80, 100)).reshape(2, 2, 3, 80, 100)
    assert_array_equal(cut[..., 0, 0], [[[20., 1020., 2020.], [120., 1120., 2120.]],
                                        [[220., 1220., 2220.], [320., 1320., 2320.]]])
    assert (numpy.diff(cut, axis=-1) == 1.).all()
    assert (numpy.diff(cut, axis=-2) == 2.).all()
