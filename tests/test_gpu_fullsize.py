"""Size-independent properties at the benchmark's full shapes (8 x 517^2 slices,
128^2 probe x 4 modes, 4096 positions, mini-batches of 256), where the numpy
oracle would take minutes per mini-batch:
  - the far-field intensity scales with |c|^2 when the probe is scaled by c;
  - for a transparent object (O = 1) and propagators without band limit the total
    intensity of each pattern equals the probe's total intensity (unitary
    propagation, shift filter and far-field transform);
  - an LSQ-ML step with zero object / probe step sizes leaves them unchanged,
    and a full iteration keeps object, probe and positions finite."""
import numpy
import pytest
import torch

from phaser_b200 import _lib
from phaser_b200.device import DeviceEngine
from phaser_b200.synthetic import lsqml_multislice_config

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def full():
    ds = lsqml_multislice_config(seed=5)
    n = int(numpy.prod(ds.scan.shape[:-1]))
    pats = torch.ones((n, 128, 128), dtype=torch.float32, device='cuda')

    def engine(probe=None, obj=None, bwlim_frac=2 / 3):
        return DeviceEngine(probe=ds.probe if probe is None else probe, obj=ds.true_object if obj is None else obj,
                            scan=ds.scan, patterns=None, mask=ds.mask, probe_sampling=ds.probe_sampling,
                            obj_sampling=ds.obj_sampling, thicknesses=ds.thicknesses, wavelength=ds.wavelength,
                            group_max=256, patterns_on_device=pats, bwlim_frac=bwlim_frac)
    return ds, engine, n


def test_intensity_scales_with_probe_amplitude(full):
    ds, engine, n = full
    idx = numpy.random.default_rng(1).permutation(n)[:256].astype(numpy.int64)
    e1, e2 = engine(), engine(probe=(ds.probe * numpy.float32(1.5)).astype(numpy.complex64))
    g1, _ = e1.group_tensor([idx])
    g2, _ = e2.group_tensor([idx])
    i1, i2 = e1.simulate(g1[0], 256), e2.simulate(g2[0], 256)
    assert torch.allclose(i2, 2.25 * i1, rtol=1e-5, atol=1e-6 * float(i1.max()))


def test_transparent_object_conserves_probe_intensity(full):
    ds, engine, n = full
    e = engine(obj=numpy.ones_like(ds.true_object), bwlim_frac=None)   # no band limit: propagation is unitary
    idx = numpy.arange(256, dtype=numpy.int64)
    g, _ = e.group_tensor([idx])
    inten = e.simulate(g[0], 256).double().sum(dim=(1, 2))
    ref = float(numpy.sum(numpy.abs(ds.probe.astype(numpy.complex128)) ** 2))
    assert torch.allclose(inten, torch.full_like(inten, ref), rtol=1e-5)


def test_zero_step_sizes_leave_state_unchanged_and_iteration_is_finite(full):
    ds, engine, n = full
    e = engine(obj=ds.init_object)
    idx = numpy.random.default_rng(2).permutation(n)[:256].astype(numpy.int64)
    g, _ = e.group_tensor([idx])
    obj0, probe0 = e.object.clone(), e.probe.clone()
    flags = _lib.PHB_FLAG_UPDATE_OBJECT | _lib.PHB_FLAG_UPDATE_PROBE
    e.status.fill_(-1)
    e.step('lsqml', g[0], 256, flags=flags, beta_object=0.0, beta_probe=0.0)
    torch.cuda.synchronize()
    assert torch.equal(e.object, obj0) and torch.equal(e.probe, probe0)
    e.step('lsqml', g[0], 256, flags=flags | _lib.PHB_FLAG_UPDATE_POSITION, beta_object=1.0, beta_probe=1.0)
    torch.cuda.synchronize()
    assert int(e.status.cpu()[0]) == -1
    assert bool(torch.isfinite(torch.view_as_real(e.object)).all())
    assert not torch.equal(e.object, obj0)
