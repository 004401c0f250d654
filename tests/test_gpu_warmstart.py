"""The learned warm start: the network trained by this library's own kernels on
patterns its forward model simulates (multislice LSQ-ML geometry: 128^2 probe,
4 modes, 300 kV, 200 A defocus), what it gains over the flat start, and the
fallback to the flat start.

- training lowers the loss;
- on held-out random-lattice positions the trained network's patch error is
  well below the flat start's (predicting transmission 1): < 0.6 of it;
- on a held-out object the warm start passes its own residual test and is
  closer to the true object than the flat start (NRMSE of the projected
  object);
- the object handed to LSQ-ML is the candidate with the smaller pattern
  residual (warm or flat), a rejected warm start leaves the run identical to
  the plain one, and the reconstruction from it stays finite."""
import numpy
import pytest
import torch

from phaser_b200 import warmstart as WS
from phaser_b200.synthetic import simulate_patterns

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def trained():
    # the benchmark's training run (200,704 patterns, 16 epochs, about a minute): the
    # network learns the mean phase of a patch within an epoch or two and the structure
    # of the patch only later, so a shorter run does not show the gain on whole objects
    f, t = WS.training_set(196, seed=7)
    net = WS.WarmStartNet(seed=0)
    losses = net.train(f, t, epochs=16, batch=256, lr=5e-4)
    return net, losses


@pytest.fixture(scope='module')
def held_out():
    ds = next(WS.random_lattice_objects(1, seed=555, scan=32, slices=(4, 4), peak=(0.3, 0.3), spacing=(10, 10)))
    pats = simulate_patterns(ds, seed=21, device='cuda')
    return ds, pats


def lsqml_factory(ds, pats):
    from phaser_b200.engines.conventional import ConventionalEngine
    from phaser_b200.plan import ConventionalEnginePlan
    from phaser_b200.sampling import Sampling
    from phaser_b200.state import IterState, ObjectState, Patterns, ProbeState, ReconsState
    N = ds.probe.shape[-1]
    init = ds.init_object.copy()

    def make():
        state = ReconsState(iter=IterState(), wavelength=ds.wavelength,
                            probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling), ds.probe.copy()),
                            object=ObjectState(ds.obj_sampling, init.copy(), ds.thicknesses.copy()),
                            scan=ds.scan.copy())
        props = ConventionalEnginePlan(noise_model={'type': 'amplitude'}, solver={'type': 'lsqml'}, niter=10,
                                       grouping=256)
        e = ConventionalEngine({'data': Patterns(None, ds.mask), 'state': state, 'dtype': numpy.float32,
                                'seed': 'warm-start-test', 'recons_name': 'ws'}, props, patterns_on_device=pats)
        e.presolve()
        return e
    return make


def test_training_lowers_loss_and_beats_flat_start(trained):
    net, losses = trained
    assert losses[-1] < losses[0]
    fh, th = WS.training_set(4, seed=99)
    pred = net.predict(fh)
    mse_net = float(torch.mean((pred - th) ** 2))
    mse_flat = float(torch.mean(th ** 2))
    print(f"\nheld-out patch MSE: network {mse_net:.4f}, flat start {mse_flat:.4f}; training {losses}")
    assert mse_net < 0.6 * mse_flat


def test_stitched_warm_start_is_closer_than_flat(trained, held_out):
    from phaser_b200.constraints import RemovePhaseRamp
    from phaser_b200.metrics import object_nrmse
    net, _ = trained
    ds, pats = held_out
    eng = lsqml_factory(ds, pats)().eng
    obj, info = WS.warm_start_object(net, eng, pats, ds.scan)
    crop = RemovePhaseRamp(eng, None, None)
    ref = torch.from_numpy(ds.true_object).cuda()
    e_warm = object_nrmse(obj, ref, crop.rows, crop.cols)
    e_flat = object_nrmse(eng.object, ref, crop.rows, crop.cols)
    print(f"\nheld-out object NRMSE: warm start {e_warm:.4f}, flat {e_flat:.4f}; {info}")
    assert info['used']
    assert e_warm < 0.95 * e_flat


def test_warm_start_uses_the_better_fit_and_falls_back_otherwise(trained, held_out):
    net, _ = trained
    ds, pats = held_out
    make = lsqml_factory(ds, pats)
    cmp = WS.compare_with_plain(net, make, ds.true_object, pats, ds.scan, iters=3)
    info = cmp['warm']['fallback_test']
    print(f"\nwarm start: {info}; NRMSE warm {cmp['warm']['curve']} plain {cmp['plain']['curve']}")
    assert info['used'] == (info['residual_warm'] < info['residual_flat'])
    assert info['scale'] in (1.0, 1.25, 1.5)
    if not info['used']:   # fallback: identical start and identical run
        assert cmp['warm']['curve'] == pytest.approx(cmp['plain']['curve'], rel=1e-6)
    assert all(numpy.isfinite(cmp['warm']['curve']))


def test_a_rejected_warm_start_keeps_the_flat_object(trained, held_out):
    net, _ = trained
    ds, pats = held_out
    eng = lsqml_factory(ds, pats)().eng
    flat = eng.object.clone()
    # a scale so large that the candidate's simulated patterns cannot fit
    obj, info = WS.warm_start_object(net, eng, pats, ds.scan, scales=(60.0,))
    assert not info['used'] and info['residual_warm'] > info['residual_flat']
    assert torch.equal(obj, flat)


def test_uint16_patterns_give_the_same_warm_start(trained, held_out):
    """Counts held as uint16 (the resident format for large scans) give the warm start
    of the same counts in float32."""
    net, _ = trained
    ds, pats = held_out
    assert float(pats.max()) < 65536 and torch.equal(pats, torch.round(pats))
    e32 = lsqml_factory(ds, pats)().eng
    o32, i32 = WS.warm_start_object(net, e32, pats, ds.scan)
    p16 = pats.to(torch.int32).to(torch.int16).view(torch.uint16)    # same bits as a uint16 cast
    e16 = lsqml_factory(ds, p16)().eng
    o16, i16 = WS.warm_start_object(net, e16, p16, ds.scan)
    assert i16['used'] == i32['used'] and i16['scale'] == i32['scale']
    assert torch.allclose(o16, o32, rtol=1e-6, atol=1e-6)
