"""The numpy restatement of phaser.execute.prepare_for_engine against the
reference's own outputs (tests/golden/prepare.npz, made by running the
reference through make_golden.py) and scipy.ndimage.affine_transform."""
import numpy
import pytest
import scipy.ndimage

from oracle import prepare_np as PR

from .test_oracle_golden import load, rel_l2

PLANS = {
    'pad_crop_up': dict(sim_shape=(40, 40), resize_method='pad_crop', probe_modes=2),
    'pad_crop_down': dict(sim_shape=(24, 24), resize_method='pad_crop', probe_modes=2),
    'resample_up': dict(sim_shape=(36, 36), resize_method='resample', probe_modes=2),
    'resample_down': dict(sim_shape=(28, 28), resize_method='resample', probe_modes=2, obj_pad_px=9.0),
    'modes_down': dict(probe_modes=1),
    'modes_up': dict(probe_modes=4, base_mode_power=0.6),
    'reslice': dict(probe_modes=2, slices=[10.0] * 5),
    'reslice_total': dict(probe_modes=2, slices=[20.0, 20.0]),
    'to_single': dict(probe_modes=2, slices=[]),
}


def grid_of(g):
    return PR.ObjGrid(g['osamp_shape'], g['obj_sampling'], g['corner'], g['region_min'], g['region_max'])


@pytest.mark.parametrize('cval', [0.0, 1.0 + 0.5j])
@pytest.mark.parametrize('matrix,offset,shape', [((1.0, 1.0), (-3.0, 2.0), (20, 25)),
                                                  ((0.8, 1.25), (0.4, -2.3), (23, 17)),
                                                  ((1.6, 0.7), (-4.5, 3.25), (14, 30))])
def test_affine_linear_matches_scipy(matrix, offset, shape, cval):
    rng = numpy.random.default_rng(1)
    a = (rng.normal(size=(2, 19, 21)) + 1j * rng.normal(size=(2, 19, 21))).astype(numpy.complex64)
    ours = PR.affine_linear(a, matrix, offset, shape, cval)
    for k in range(2):
        ref = scipy.ndimage.affine_transform(a[k], numpy.asarray(matrix), offset=offset, output_shape=shape,
                                             order=1, mode='grid-constant', cval=cval)
        assert rel_l2(ours[k], ref) < 1e-6


@pytest.mark.parametrize('name', list(PLANS))
def test_prepare_for_engine_matches_reference(name):
    g = load('prepare.npz')
    grid = grid_of(g)
    kw = dict(PLANS[name])
    if 'slices' in kw:
        kw['slices'] = numpy.asarray(kw['slices'], numpy.float32)
    pats, mask, probe, psamp, obj, grid2, thick = PR.prepare_for_engine(
        g['patterns'], g['mask'], g['probe'], g['probe_sampling'], g['object'], grid, g['thicknesses'], g['scan'],
        **kw)
    p = name + '__'
    assert numpy.allclose(psamp, g[p + 'probe_sampling'], rtol=1e-12)
    assert numpy.array_equal(grid2.shape, g[p + 'obj_shape'])
    assert numpy.allclose(grid2.sampling, g[p + 'obj_sampling'], rtol=1e-12)
    assert numpy.allclose(grid2.corner, g[p + 'corner'], rtol=1e-12, atol=1e-12)
    assert numpy.allclose(grid2.region_min, g[p + 'region_min']) and numpy.allclose(grid2.region_max, g[p + 'region_max'])
    assert numpy.allclose(thick, g[p + 'thicknesses'])
    assert probe.shape == g[p + 'probe'].shape and rel_l2(probe, g[p + 'probe']) < 1e-5
    ref_obj = g[p + 'object'] if (p + 'object') in g else g['object']
    assert obj.shape == ref_obj.shape and rel_l2(obj, ref_obj) < 1e-5
    ref_pats = g[p + 'patterns'] if (p + 'patterns') in g else g['patterns']
    assert pats.shape == ref_pats.shape and rel_l2(pats, ref_pats) < 1e-5
    ref_mask = g[p + 'mask'] if (p + 'mask') in g else g['mask']
    assert rel_l2(mask, ref_mask) < 1e-5


@pytest.mark.parametrize('align', ['top', 'middle', 'bottom'])
@pytest.mark.parametrize('pad', ['vacuum', 'edge', 'average'])
def test_resample_slices_matches_reference(align, pad):
    g = load('prepare.npz')
    obj = g['object'][:, 20:32, 24:36]
    out = PR.resample_slices(obj, g['thicknesses'], [12.0, 9.0, 14.0, 11.0], align, pad)
    assert rel_l2(out, g[f'slices_{align}_{pad}']) < 1e-5


def test_product_grid_arithmetic_matches_reference():
    """The host grid steps of phaser_b200.prepare (ObjectSampling.with_sampling and
    expand_to_scan, the slices specifications) give the reference's grids."""
    from phaser_b200 import plan as PL
    from phaser_b200.sampling import ObjectSampling
    g = load('prepare.npz')
    grid = ObjectSampling(tuple(g['osamp_shape']), g['obj_sampling'], g['corner'], g['region_min'], g['region_max'])
    N = numpy.asarray(g['probe'].shape[-2:])
    psamp = numpy.asarray(g['probe_sampling'])
    for name, shape, method, pad in (('pad_crop_up', 40, 'pad_crop', 5.0), ('resample_down', 28, 'resample', 9.0)):
        new_samp = psamp * N / shape if method == 'pad_crop' else psamp
        g2 = grid.with_sampling(new_samp) if not numpy.allclose(new_samp, grid.sampling) else grid
        g2 = g2.expand_to_scan(g['scan'], new_samp * shape / 2. + pad * new_samp)
        p = name + '__'
        assert numpy.array_equal(g2.shape, g[p + 'obj_shape'])
        assert numpy.allclose(g2.corner, g[p + 'corner'], rtol=1e-12, atol=1e-12)
        assert numpy.allclose(g2.region_min, g[p + 'region_min']) and numpy.allclose(g2.region_max, g[p + 'region_max'])
    assert grid.expand_to_scan(g['scan'], psamp * N / 2. + 5.0 * psamp) == grid   # already covers the scan
    assert PL.slice_thicknesses(PL.SliceStep(n=5, slice_thickness=10.0)) == [10.0] * 5
    assert PL.slice_thicknesses({'n': 2, 'total_thickness': 40.0}) == [20.0, 20.0]
    assert PL.slice_thicknesses({'thicknesses': [1, 2]}) == [1.0, 2.0]
    assert PL.slice_thicknesses(PL.SliceList(thicknesses=[])) == [] and PL.slice_thicknesses(None) is None
    with pytest.raises(ValueError):
        PL.slice_thicknesses({'n': 3})


def test_tilt_map_rule():
    """A gradient plan whose solvers name 'tilt' gets a zero tilt map (execute.py:396-400)."""
    from phaser_b200 import plan as PL
    from phaser_b200.prepare import solves_for_tilt
    assert solves_for_tilt(PL.GradientEnginePlan(solvers={'object': {'type': 'adam'}, 'tilt': {'type': 'sgd'}}))
    assert solves_for_tilt(PL.GradientEnginePlan(solvers={'positions,tilt': {'type': 'sgd'}}))
    assert solves_for_tilt(PL.GradientEnginePlan(solvers={frozenset({'tilt'}): {'type': 'sgd'}}))
    assert not solves_for_tilt(PL.GradientEnginePlan(solvers={'object': {'type': 'adam'}}))
    assert not solves_for_tilt(PL.ConventionalEnginePlan())
