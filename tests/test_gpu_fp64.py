"""Error of the complex64 B200 kernels against the float64 oracle.

The kernels compute in complex64 with float64 only in the step-size and
normalisation sums; these tests state their error against the same algorithm
evaluated in float64/complex128 (and, for scale, the error of the oracle's own
complex64 evaluation):
  forward model (far-field intensity)         < 1e-5 relative L2
  one LSQ-ML mini-batch: object, probe        < 1e-5 relative L2 (updates < 1e-3)
  gradient-engine loss / object gradient      < 1e-5 / 1e-4
Run with -s to print the measured values."""
import numpy
import pytest
import torch

from oracle import phaser_np as P
from phaser_b200 import _lib
from phaser_b200.device import DeviceEngine, NoiseSpec

from .cases import make_case
from .test_gpu_engine import rel_l2

pytestmark = pytest.mark.gpu


def f64_inputs(c):
    N = c.probe.shape[-1]
    ky, kx = P.recip_grid((N, N), c.probe_sampling, numpy.float64)
    g = P.Geometry(numpy.asarray(c.osamp.corner), numpy.asarray(c.osamp.sampling), ky, kx, c.thick)
    props = P.make_propagators(ky, kx, c.probe_sampling, c.wavelength, c.thick.astype(numpy.float64))
    return (g, c.probe.astype(numpy.complex128), c.obj.astype(numpy.complex128), props,
            c.patterns.reshape(-1, N, N).astype(numpy.float64), c.mask.astype(numpy.float64))


def engine(c, B, noise=NoiseSpec()):
    return DeviceEngine(probe=c.probe, obj=c.obj, scan=c.scan, patterns=c.patterns, mask=c.mask,
                        probe_sampling=c.probe_sampling, obj_sampling=c.osamp, thicknesses=c.thick,
                        wavelength=c.wavelength, noise=noise, group_max=B)


def test_forward_model_error_vs_float64():
    c = make_case(seed=301, N=128, M=4, S=4, scan_shape=(3, 3))
    n = 9
    eng = engine(c, n)
    gt, sizes = eng.group_tensor([numpy.arange(n, dtype=numpy.int64)])
    sim = eng.simulate(gt[0], sizes[0]).cpu().numpy()
    g, probe, obj, props, _, _ = f64_inputs(c)
    flat = c.scan.reshape(-1, 2)
    psi0, cuts, _, _ = P.cutout_group(g, probe, obj, flat)
    psi = P._forward(psi0, cuts, P.tilt_propagators(g.ky, g.kx, c.thick, props, None))
    ref = numpy.sum(P.abs2(P.fft2c(psi[-1] * cuts[:, -1, None])), axis=1)
    # the oracle's own complex64 evaluation, for scale
    g32 = c.geom()
    p0, ct, _, _ = P.cutout_group(g32, c.probe, c.obj, flat)
    ps = P._forward(p0, ct, P.tilt_propagators(g32.ky, g32.kx, c.thick, c.props(), None))
    own = numpy.sum(P.abs2(P.fft2c(ps[-1] * ct[:, -1, None])), axis=1)
    err, err_np = rel_l2(sim, ref), rel_l2(own, ref)
    print(f"\nforward model vs float64: B200 {err:.2e}, numpy complex64 {err_np:.2e}")
    assert err < 1e-5


def test_lsqml_step_error_vs_float64():
    c = make_case(seed=302, N=128, M=4, S=4, scan_shape=(3, 3))
    idx = numpy.arange(9, dtype=numpy.int64)
    eng = engine(c, 9)
    gt, sizes = eng.group_tensor([idx])
    flags = (_lib.PHB_FLAG_UPDATE_OBJECT | _lib.PHB_FLAG_UPDATE_PROBE | _lib.PHB_FLAG_UPDATE_POSITION
             | _lib.PHB_FLAG_CALC_ERROR)
    eng.status.fill_(-1)
    eng.step('lsqml', gt[0], sizes[0], flags=flags, beta_object=0.9, beta_probe=0.8)
    probe_g, obj_g, _ = eng.host_state()
    g, probe, obj, props, pats, mask = f64_inputs(c)
    ref = P.lsqml_group(g, probe, obj, c.scan.reshape(-1, 2).astype(numpy.float64), pats, mask, props, None,
                        P.NoiseModel(), P.LSQMLParams(0.9, 0.8, 1e-2, 1e-2, 1e-4), update_position=True)
    e_obj, e_probe = rel_l2(obj_g, ref['object']), rel_l2(probe_g, ref['probe'])
    d_obj = rel_l2(obj_g - c.obj, ref['object'] - obj)
    d_probe = rel_l2(probe_g - c.probe, ref['probe'] - probe)
    print(f"\nLSQ-ML step vs float64: object {e_obj:.2e} (update {d_obj:.2e}), probe {e_probe:.2e} "
          f"(update {d_probe:.2e})")
    assert e_obj < 1e-5 and e_probe < 1e-5
    assert d_obj < 1e-3 and d_probe < 1e-3


def test_gradient_error_vs_float64():
    c = make_case(seed=303, N=128, M=2, S=4, scan_shape=(3, 3))
    idx = numpy.arange(9, dtype=numpy.int64)
    eng = engine(c, 9, NoiseSpec('poisson', 1e-3, 0.0, 0.1))
    gt, sizes = eng.group_tensor([idx])
    g_obj = torch.zeros_like(eng.object)
    loss = torch.zeros((1,), dtype=torch.float64, device='cuda')
    eng.status.fill_(-1)
    eng.step('grad', gt[0], sizes[0], flags=_lib.PHB_FLAG_UPDATE_OBJECT, grad_object=g_obj, group_loss=loss)
    g, probe, obj, props, pats, mask = f64_inputs(c)
    L, r_obj, _, _ = P.grad_model_grads(g, probe, obj, c.scan.reshape(-1, 2).astype(numpy.float64), pats, mask,
                                        props, None, P.NoiseModel(kind='poisson', eps=1e-3))
    e_loss = abs(float(loss.cpu()[0]) - float(L)) / abs(float(L))
    e_grad = rel_l2(g_obj.cpu().numpy(), r_obj)
    print(f"\ngradient engine vs float64: loss {e_loss:.2e}, object gradient {e_grad:.2e}")
    assert e_loss < 1e-5 and e_grad < 1e-4
