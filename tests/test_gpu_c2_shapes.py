"""Parity at the shapes of the multislice LSQ-ML benchmark: probe 128^2 with 4
incoherent modes (70/15/10/5 %), 8 slices of 2 nm, 300 kV, 25 mrad, 200 A defocus,
6 px scan step, Gaussian-atom lattice objects at 0.2 rad per slice, Poisson data
at 1e6 e- per pattern.

  * one LSQ-ML and one ePIE mini-batch of 64 positions on the full benchmark
    object grid (518^2, scan 64 x 64), from a partly reconstructed object, against
    the numpy oracle (complex64) and the float64 oracle;
  * one gradient-engine loss + adjoint on the same group against the oracle's
    hand-written adjoint (complex64 and float64);
  * three whole LSQ-ML iterations at batch 256 (momentum position correction)
    on a 16 x 16 scan of the same optics, compared after EVERY iteration with
    the complex64 oracle and the float64 oracle (phaser/engines/conventional/
    run.py:15-123 with solvers.py:171-290 semantics).

Tolerances as in the smaller parity tests: a mini-batch's object / probe within
1e-5 relative L2 (their updates within 1e-3), per-position errors within 1e-4,
position steps within 2e-3; whole iterations within 1e-4.  The float64 figures
are printed (pytest -s) and bounded by the same limits."""
import numpy
import pytest
import torch

from oracle import phaser_np as P
from phaser_b200 import _lib
from phaser_b200 import plan as PL
from phaser_b200.device import DeviceEngine, NoiseSpec
from phaser_b200.engines.conventional import ConventionalEngine
from phaser_b200.sampling import Sampling
from phaser_b200.state import ReconsState, ProbeState, ObjectState, IterState, Patterns
from phaser_b200.synthetic import lsqml_multislice_config

from .test_gpu_engine import rel_l2

pytestmark = pytest.mark.gpu


def oracle_patterns(ds, idx, seed):
    """Noisy far-field patterns of scan rows `idx` from the oracle's complex64 forward
    model (probe and true object of the dataset), Poisson at the dataset's dose."""
    N = ds.probe.shape[-1]
    ky, kx = P.recip_grid((N, N), ds.probe_sampling, numpy.float32)
    g = P.Geometry(numpy.asarray(ds.obj_sampling.corner), numpy.asarray(ds.obj_sampling.sampling), ky, kx,
                   ds.thicknesses)
    props = P.make_propagators(ky, kx, ds.probe_sampling, ds.wavelength, ds.thicknesses)
    flat = ds.scan.reshape(-1, 2)[idx]
    psi0, cuts, _, _ = P.cutout_group(g, ds.probe, ds.true_object, flat)
    psi = P._forward(psi0, cuts, P.tilt_propagators(ky, kx, ds.thicknesses, props, None))
    inten = numpy.sum(P.abs2(P.fft2c(psi[-1] * cuts[:, -1, None])), axis=1)
    inten *= ds.counts / inten.sum(axis=(1, 2), keepdims=True)
    return (numpy.random.default_rng(seed).poisson(inten)).astype(numpy.float32)


def geometry(ds, dtype):
    N = ds.probe.shape[-1]
    ky, kx = P.recip_grid((N, N), ds.probe_sampling, dtype)
    g = P.Geometry(numpy.asarray(ds.obj_sampling.corner), numpy.asarray(ds.obj_sampling.sampling), ky, kx,
                   ds.thicknesses)
    props = P.make_propagators(ky, kx, ds.probe_sampling, ds.wavelength,
                               ds.thicknesses.astype(dtype))
    return g, props


@pytest.fixture(scope='module')
def c2_group():
    """Benchmark dataset (518^2 x 8 slices), 64 positions spread over the scan, their
    patterns, the probe after the presolve rescale (so the step sizes are those of a
    real run), and a partly reconstructed estimate (60 % of each slice's true phase, 97 %
    amplitude): from the flat start the position gradient is rounding noise (the
    object has no structure yet), and its parity would be meaningless."""
    ds = lsqml_multislice_config(seed=7)
    n = int(numpy.prod(ds.scan.shape[:-1]))
    idx = numpy.sort(numpy.random.default_rng(8).choice(n, 64, replace=False)).astype(numpy.int64)
    pats = oracle_patterns(ds, idx, 9)
    est = (0.97 * numpy.exp(0.6j * numpy.angle(ds.true_object))).astype(numpy.complex64)
    g, props = geometry(ds, numpy.float32)
    f = P.epie_dry_run(g, ds.probe, est, ds.scan.reshape(-1, 2)[idx], pats, ds.mask, props, None)
    probe = (ds.probe * numpy.sqrt(numpy.mean(f))).astype(numpy.complex64)
    return ds, idx, pats, probe, est


@pytest.mark.parametrize('solver', ['lsqml', 'epie'])
def test_c2_group_matches_oracle_and_float64(c2_group, solver):
    ds, idx, pats, probe, est = c2_group
    N = ds.probe.shape[-1]
    n = int(numpy.prod(ds.scan.shape[:-1]))
    full = numpy.zeros((n, N, N), numpy.float32)
    full[idx] = pats
    eng = DeviceEngine(probe=probe, obj=est, scan=ds.scan, patterns=full, mask=ds.mask,
                       probe_sampling=ds.probe_sampling, obj_sampling=ds.obj_sampling,
                       thicknesses=ds.thicknesses, wavelength=ds.wavelength, group_max=len(idx))
    gt, sizes = eng.group_tensor([idx])
    flags = (_lib.PHB_FLAG_UPDATE_OBJECT | _lib.PHB_FLAG_UPDATE_PROBE | _lib.PHB_FLAG_UPDATE_POSITION
             | _lib.PHB_FLAG_CALC_ERROR)
    eng.status.fill_(-1)
    if solver == 'lsqml':
        params = P.LSQMLParams(0.9, 0.8, 1e-2, 1e-2, 1e-4)
        eng.step('lsqml', gt[0], sizes[0], flags=flags, beta_object=0.9, beta_probe=0.8,
                 illum_reg_object=1e-2, illum_reg_probe=1e-2, gamma=1e-4)
        fn = P.lsqml_group
    else:
        params = P.EPIEParams(0.9, 0.8)
        eng.step('epie', gt[0], sizes[0], flags=flags, beta_object=0.9, beta_probe=0.8)
        fn = P.epie_group
    p_gpu, o_gpu, _ = eng.host_state()
    assert int(eng.status.cpu()[0]) == -1
    err_gpu = eng.errors.cpu().numpy()[idx]
    pos_gpu = eng.pos_update.cpu().numpy()[idx]
    scan = ds.scan.reshape(-1, 2)[idx]
    g32, props32 = geometry(ds, numpy.float32)
    ref = fn(g32, probe, est, scan, pats, ds.mask, props32, None, P.NoiseModel(), params,
             update_position=True)
    g64, props64 = geometry(ds, numpy.float64)
    r64 = fn(g64, probe.astype(numpy.complex128), est.astype(numpy.complex128),
             scan.astype(numpy.float64), pats.astype(numpy.float64), ds.mask.astype(numpy.float64), props64, None,
             P.NoiseModel(), params, update_position=True)
    e_obj, e_probe = rel_l2(o_gpu, ref['object']), rel_l2(p_gpu, ref['probe'])
    d_obj = rel_l2(o_gpu - est, ref['object'] - est)
    d_probe = rel_l2(p_gpu - probe, ref['probe'] - probe)
    f_obj, f_probe = rel_l2(o_gpu, r64['object']), rel_l2(p_gpu, r64['probe'])
    n_obj = rel_l2(ref['object'], r64['object'])
    print(f"\n{solver} 64 positions, N=128 M=4 S=8, 518^2: vs oracle object {e_obj:.2e} (update {d_obj:.2e}), "
          f"probe {e_probe:.2e} (update {d_probe:.2e}); vs float64 object {f_obj:.2e}, probe {f_probe:.2e} "
          f"(numpy complex64 vs float64: object {n_obj:.2e})")
    assert e_obj < 1e-5 and e_probe < 1e-5
    assert d_obj < 1e-3 and d_probe < 1e-3
    assert f_obj < 1e-5 and f_probe < 1e-5
    p64 = rel_l2(pos_gpu, r64['pos_update'])
    print(f"position step vs oracle {rel_l2(pos_gpu, ref['pos_update']):.2e}, vs float64 {p64:.2e} "
          f"(numpy complex64 vs float64 {rel_l2(ref['pos_update'], r64['pos_update']):.2e})")
    assert numpy.allclose(err_gpu, ref['errors'], rtol=1e-4)
    assert rel_l2(pos_gpu, ref['pos_update']) < 2e-3
    assert p64 < 2e-3


def test_c2_gradient_group_matches_oracle_and_float64(c2_group):
    """The gradient engine's fused loss + adjoint on the same 64 positions of the benchmark
    dataset (amplitude noise model): loss, object / probe / position gradients against the
    oracle's hand-written adjoint in complex64 and float64."""
    ds, idx, pats, probe, est = c2_group
    N = ds.probe.shape[-1]
    n = int(numpy.prod(ds.scan.shape[:-1]))
    full = numpy.zeros((n, N, N), numpy.float32)
    full[idx] = pats
    eng = DeviceEngine(probe=probe, obj=est, scan=ds.scan, patterns=full, mask=ds.mask,
                       probe_sampling=ds.probe_sampling, obj_sampling=ds.obj_sampling,
                       thicknesses=ds.thicknesses, wavelength=ds.wavelength, group_max=len(idx),
                       noise=NoiseSpec('amplitude', 1e-2, 0.0, 0.1))
    gt, sizes = eng.group_tensor([idx])
    g_obj, g_probe, g_pos = torch.zeros_like(eng.object), torch.zeros_like(eng.probe), torch.zeros_like(eng.scan)
    total = torch.zeros((1,), dtype=torch.float64, device=eng.device)
    eng.status.fill_(-1)
    eng.step('grad', gt[0], sizes[0],
             flags=_lib.PHB_FLAG_UPDATE_OBJECT | _lib.PHB_FLAG_UPDATE_PROBE | _lib.PHB_FLAG_UPDATE_POSITION,
             grad_object=g_obj, grad_probe=g_probe, grad_pos=g_pos, group_loss=total)
    torch.cuda.synchronize()
    assert int(eng.status.cpu()[0]) == -1
    scan = ds.scan.reshape(-1, 2)[idx]
    g32, props32 = geometry(ds, numpy.float32)
    L, r_obj, r_probe, r_pos = P.grad_model_grads(g32, probe, est, scan, pats, ds.mask, props32, None,
                                                 P.NoiseModel(eps=1e-2))
    g64, props64 = geometry(ds, numpy.float64)
    L64, f_obj, f_probe, f_pos = P.grad_model_grads(
        g64, probe.astype(numpy.complex128), est.astype(numpy.complex128), scan.astype(numpy.float64),
        pats.astype(numpy.float64), ds.mask.astype(numpy.float64), props64, None, P.NoiseModel(eps=1e-2))
    go, gp, gs = g_obj.cpu().numpy(), g_probe.cpu().numpy(), g_pos.cpu().numpy()[idx]
    print(f"\ngradient 64 positions, N=128 M=4 S=8: loss {float(total.cpu()[0]):.6e} vs oracle {float(L):.6e} "
          f"vs float64 {float(L64):.6e}; object gradient vs oracle {rel_l2(go, r_obj):.2e}, vs float64 "
          f"{rel_l2(go, f_obj):.2e}; probe {rel_l2(gp, r_probe):.2e} / {rel_l2(gp, f_probe):.2e}; "
          f"positions {rel_l2(gs, r_pos):.2e} / {rel_l2(gs, f_pos):.2e}")
    assert float(total.cpu()[0]) == pytest.approx(float(L), rel=1e-5)
    # the loss is a float32 sum of 64 x 128^2 terms: numpy's complex64 evaluation is 9e-6 from
    # float64 itself
    assert float(total.cpu()[0]) == pytest.approx(float(L64), rel=5e-5)
    assert rel_l2(go, r_obj) < 1e-4 and rel_l2(go, f_obj) < 1e-4
    assert rel_l2(gp, r_probe) < 1e-4 and rel_l2(gp, f_probe) < 1e-4
    assert rel_l2(gs, r_pos) < 2e-3 and rel_l2(gs, f_pos) < 2e-3


def test_c2_lsqml_iterations_match_oracle_and_float64():
    """Three whole LSQ-ML iterations, batch 256, 16 x 16 scan of the benchmark optics:
    presolve, sparse shuffled groups, momentum position correction; object, probe and
    scan compared with the complex64 and float64 oracles after every iteration."""
    ds = lsqml_multislice_config(seed=11, scan=16)
    N = ds.probe.shape[-1]
    n = int(numpy.prod(ds.scan.shape[:-1]))
    pats = oracle_patterns(ds, numpy.arange(n), 12).reshape(*ds.scan.shape[:-1], N, N)
    niter, seed = 3, 'c2-iterations'
    props = PL.ConventionalEnginePlan(
        noise_model={'type': 'amplitude'}, solver={'type': 'lsqml'},
        position_solver={'type': 'momentum', 'step_size': 1e-3, 'max_step_size': 0.2, 'momentum': 0.9},
        niter=niter, grouping=256, update_positions=True, calc_error_fraction=1.0)
    state = ReconsState(iter=IterState(), wavelength=ds.wavelength,
                        probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling), ds.probe.copy()),
                        object=ObjectState(ds.obj_sampling, ds.init_object.copy(), ds.thicknesses.copy()),
                        scan=ds.scan.copy())
    e = ConventionalEngine({'data': Patterns(pats, ds.mask), 'state': state, 'dtype': numpy.float32,
                            'seed': seed, 'recons_name': 'c2'}, props)
    e.presolve()
    gpu = []
    for i in range(1, niter + 1):
        e.iteration(i)
        gpu.append(e.eng.host_state())

    def oracle(dtype):
        cdt = numpy.complex128 if dtype == numpy.float64 else numpy.complex64
        run = P.ConventionalRun(solver='lsqml', niter=niter, grouping=256, seed=seed, noise=P.NoiseModel(),
                                lsqml=P.LSQMLParams(1.0, 1.0, 1e-2, 1e-2, 1e-4), update_positions=True,
                                position_solver='momentum', pos_step_size=1e-3, pos_max_step=0.2,
                                pos_momentum=0.9, calc_error_fraction=1.0)
        out = []
        P.run_conventional(run, probe=ds.probe.astype(cdt), obj=ds.init_object.astype(cdt),
                           scan=ds.scan.astype(dtype), patterns=pats.astype(dtype), mask=ds.mask.astype(dtype),
                           probe_sampling=ds.probe_sampling, corner=ds.obj_sampling.corner,
                           obj_sampling=ds.obj_sampling.sampling, thicknesses=ds.thicknesses.astype(dtype),
                           wavelength=ds.wavelength,
                           iteration_callback=lambda it, p, o, s, err: out.append((p.copy(), o.copy(), s.copy())))
        return out

    r32, r64 = oracle(numpy.float32), oracle(numpy.float64)
    for i, ((pg, og, sg), (p32, o32, s32), (p64, o64, s64)) in enumerate(zip(gpu, r32, r64), start=1):
        e_o, e_p = rel_l2(og, o32), rel_l2(pg, p32)
        f_o, f_p = rel_l2(og, o64), rel_l2(pg, p64)
        n_o = rel_l2(o32, o64)
        ds_max = float(numpy.max(numpy.abs(sg - s32)))
        print(f"\niteration {i}: vs oracle object {e_o:.2e} probe {e_p:.2e} scan {ds_max:.1e} A; vs float64 "
              f"object {f_o:.2e} probe {f_p:.2e} (numpy complex64 vs float64 object {n_o:.2e})")
        assert e_o < 1e-4 and e_p < 1e-4
        assert f_o < 1e-4 and f_p < 1e-4
        assert ds_max < 1e-4
        assert numpy.max(numpy.abs(sg - s64)) < 1e-4
