"""Final reconstruction quality against the numpy restatement of the reference
on identical seeded inputs: the object NRMSE (against the simulated truth) of a
whole run on the GPU must be within 1 % of the same run's NRMSE in the oracle.

- the single-slice ePIE configuration as specified: 64^2 probe (20 mrad,
  200 kV, 100 A defocus), 32 x 32 scan at 4 px with +-0.5 px jitter, 1e5
  e-/pattern, grouping 64, 10 iterations;
- the multislice LSQ-ML configuration's optics and object (8 x 2 nm slices,
  128^2 probe x 4 modes, momentum position correction) on a 12 x 12 scan,
  4 iterations, so that the host oracle finishes in seconds.

The NRMSE is computed by one numpy function for both results (projected object
over the scanned region, linear phase ramps removed, global phase fitted)."""
import os

import numpy
import pytest

from oracle import phaser_np as O
from phaser_b200 import plan as PL
from phaser_b200.engines.conventional import run_engine
from phaser_b200.sampling import Sampling
from phaser_b200.state import IterState, ObjectState, Patterns, ProbeState, ReconsState
from phaser_b200.synthetic import epie_single_slice_config, lsqml_multislice_config, simulate_patterns

pytestmark = pytest.mark.gpu


def region(ds):
    os_ = ds.obj_sampling
    corner, samp = numpy.asarray(os_.corner), numpy.asarray(os_.sampling)
    lo = numpy.ceil((numpy.asarray(os_.region_min) - corner) / samp).astype(int)
    hi = (numpy.floor((numpy.asarray(os_.region_max) - corner) / samp) + 1).astype(int)
    H, W = ds.true_object.shape[-2:]
    return (max(lo[0], 0), min(hi[0], H)), (max(lo[1], 0), min(hi[1], W))


def nrmse(rec, ref, rows, cols):
    a = numpy.prod(rec, axis=0, keepdims=True).astype(numpy.complex128)
    b = numpy.prod(ref, axis=0, keepdims=True).astype(numpy.complex128)
    a = O.remove_phase_ramp(a, rows, cols)[0, rows[0]:rows[1], cols[0]:cols[1]]
    b = O.remove_phase_ramp(b, rows, cols)[0, rows[0]:rows[1], cols[0]:cols[1]]
    phi0 = numpy.angle(numpy.sum(numpy.conj(a) * b))
    return float(numpy.linalg.norm(a * numpy.exp(1j * phi0) - b) / numpy.linalg.norm(b))


CASES = {
    'single_slice_epie': dict(make=lambda: epie_single_slice_config(seed=3), solver='epie', niter=10, grouping=64,
                              positions=False),
    'multislice_lsqml': dict(make=lambda: lsqml_multislice_config(seed=4, scan=12), solver='lsqml', niter=4,
                             grouping=64, positions=True),
}


@pytest.mark.parametrize('name', list(CASES))
def test_final_nrmse_within_one_percent_of_oracle(name):
    cfg = CASES[name]
    ds = cfg['make']()
    pats = simulate_patterns(ds, seed=9, device='cuda', group=64).cpu().numpy()
    N = ds.probe.shape[-1]
    pos = dict(position_solver={'type': 'momentum', 'step_size': 1e-3, 'max_step_size': 0.2, 'momentum': 0.9},
               update_positions=True) if cfg['positions'] else {}
    props = PL.ConventionalEnginePlan(noise_model={'type': 'amplitude', 'eps': 1e-3}, solver={'type': cfg['solver']},
                                      niter=cfg['niter'], grouping=cfg['grouping'], **pos)
    state = ReconsState(iter=IterState(), wavelength=ds.wavelength,
                        probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling), ds.probe.copy()),
                        object=ObjectState(ds.obj_sampling, ds.init_object.copy(), ds.thicknesses.copy()),
                        scan=ds.scan.copy())
    out = run_engine({'data': Patterns(pats, ds.mask), 'state': state, 'dtype': numpy.float32, 'seed': 'nrmse',
                      'recons_name': name}, props)
    O.set_fft_workers(os.cpu_count() or 1)
    run = O.ConventionalRun(solver=cfg['solver'], niter=cfg['niter'], grouping=cfg['grouping'], seed='nrmse',
                            noise=O.NoiseModel(eps=1e-3), update_positions=cfg['positions'],
                            position_solver='momentum' if cfg['positions'] else None, pos_step_size=1e-3,
                            pos_max_step=0.2, pos_momentum=0.9)
    os_ = ds.obj_sampling
    _, obj_ref, _, _ = O.run_conventional(run, probe=ds.probe, obj=ds.init_object, scan=ds.scan, patterns=pats,
                                          mask=ds.mask, probe_sampling=ds.probe_sampling, corner=os_.corner,
                                          obj_sampling=os_.sampling, thicknesses=ds.thicknesses,
                                          wavelength=ds.wavelength)
    rows, cols = region(ds)
    e_gpu = nrmse(out.object.data, ds.true_object, rows, cols)
    e_ref = nrmse(obj_ref, ds.true_object, rows, cols)
    e_flat = nrmse(ds.init_object, ds.true_object, rows, cols)
    print(f"\n{name}: NRMSE flat {e_flat:.5f}, GPU {e_gpu:.5f}, oracle {e_ref:.5f}")
    assert e_gpu < e_flat                          # the run reconstructs something
    assert abs(e_gpu - e_ref) <= 0.01 * e_ref
