"""The learned warm start: the network trained by this library's own kernels on
patterns its forward model simulates, what it gains over the flat start, and
the fallback to the flat start.

- training lowers the loss;
- on held-out random-lattice positions the trained network's patch error is
  well below the flat start's (predicting transmission 1): < 0.6 of it;
- on a held-out single-slice object, the initial object handed to LSQ-ML is
  the candidate with the smaller pattern residual (warm or flat), and the
  reconstruction from it stays finite (the NRMSE curves are printed with -s)."""
import numpy
import pytest
import torch

from phaser_b200 import warmstart as WS
from phaser_b200.synthetic import epie_single_slice_config, simulate_patterns

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def trained():
    f, t = WS.training_set(48, seed=3)
    net = WS.WarmStartNet(seed=0)
    losses = net.train(f, t, epochs=2, batch=256, lr=1e-3)
    return net, losses


def test_training_lowers_loss_and_beats_flat_start(trained):
    net, losses = trained
    assert losses[-1] < losses[0]
    fh, th = WS.training_set(4, seed=99)
    pred = net.predict(fh)
    mse_net = float(torch.mean((pred - th) ** 2))
    mse_flat = float(torch.mean(th ** 2))
    print(f"\nheld-out patch MSE: network {mse_net:.4f}, flat start {mse_flat:.4f}; training {losses}")
    assert mse_net < 0.6 * mse_flat


def test_warm_start_uses_the_better_fit_and_falls_back_otherwise(trained):
    net, _ = trained
    ds = epie_single_slice_config(seed=21)
    pats = simulate_patterns(ds, seed=21, device='cuda', group=64)
    cmp = WS.compare_with_plain(net, ds, pats, iters=5)
    info = cmp['warm']['fallback_test']
    print(f"\nwarm start: {info}; initial NRMSE warm {cmp['warm']['curve'][0]:.4f} flat "
          f"{cmp['plain']['curve'][0]:.4f}; after 5 iterations warm {cmp['warm']['curve'][-1]:.4f} "
          f"plain {cmp['plain']['curve'][-1]:.4f}")
    assert info['used'] == (info['residual_warm'] < info['residual_flat'])
    if not info['used']:   # fallback: identical start and identical run
        assert cmp['warm']['curve'] == pytest.approx(cmp['plain']['curve'], rel=1e-6)
    assert all(numpy.isfinite(cmp['warm']['curve']))
