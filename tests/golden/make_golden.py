"""Generate the golden fixtures in this folder by running the REFERENCE phaser
numpy code (not the oracle) on small seeded inputs.

Run where the reference sources are available, with PHASER_REF naming the
root of the phaser source tree (required):

    PHASER_REF=<phaser source root> python tests/golden/make_golden.py

`pane` (py-pane 0.11.3) is not installed there, so `pane_shim/` supplies the
few names the reference imports.  The fixtures store inputs and outputs, so the
tests that read them never need the reference.
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy

HERE = Path(__file__).resolve().parent
REF = os.environ.get('PHASER_REF')
if not REF:
    sys.exit("set PHASER_REF to the root of the phaser source tree")
sys.path.insert(0, str(HERE / 'pane_shim'))
sys.path.insert(0, REF)

from phaser.utils.num import Sampling, fft2, ifft2  # noqa: E402
from phaser.utils.object import ObjectSampling  # noqa: E402
from phaser.utils import optics, misc, scan as scan_mod, physics  # noqa: E402
from phaser.state import (ReconsState, ProbeState, ObjectState, IterState,  # noqa: E402
                          ProgressState, Patterns)
from phaser.plan import (AmplitudeNoisePlan, AnscombeNoisePlan, PoissonNoisePlan,  # noqa: E402
                         LSQMLSolverPlan, EPIESolverPlan, ConventionalEnginePlan)
from phaser.hooks.solver import (NoiseModelHook, ConventionalSolverHook, PositionSolverHook,  # noqa: E402
                                 MomentumPositionSolverProps)
from phaser.engines.common.noise_models import (AmplitudeNoiseModel, AnscombeNoiseModel,  # noqa: E402
                                                PoissonNoiseModel)
from phaser.engines.common.simulation import (SimulationState, make_propagators,  # noqa: E402
                                              cutout_group, slice_forwards, tilt_propagators)
from phaser.engines.conventional import solvers  # noqa: E402
from phaser.engines.conventional.run import run_engine  # noqa: E402

F32, C64 = numpy.float32, numpy.complex64


def save(name: str, **arrays):
    path = HERE / name
    numpy.savez_compressed(path, **arrays)
    print(f"wrote {path.name}: {path.stat().st_size} B")


def make_case(seed: int, N: int, M: int, S: int, scan_shape, step: float,
              samp: float = 0.4, kv: float = 200e3, tilt: bool = False, dtype=F32):
    """A small reconstruction: the reference's geometry helpers build the
    probe, scan and object grid; the 'true' object makes the patterns and a
    perturbed copy is the current estimate."""
    rng = numpy.random.default_rng(seed)
    cdt = C64 if dtype == F32 else numpy.complex128
    wavelength = physics.Electron(kv).wavelength
    psamp = Sampling((N, N), sampling=(samp, samp))
    ky, kx = psamp.recip_grid(dtype=dtype, xp=numpy)
    base = optics.make_focused_probe(ky, kx, wavelength, 25., defocus=60.)
    probe = optics.make_hermetian_modes(base, M, 0.7, [0.5, 1/3, 1/6][:M - 1]) if M > 1 else base[None]
    probe = probe.astype(cdt)
    scan = scan_mod.make_raster_scan(scan_shape, step, dtype=dtype, xp=numpy)
    scan = (scan + rng.uniform(-0.3, 0.3, scan.shape) * step).astype(dtype)
    osamp = ObjectSampling.from_scan(scan, psamp.sampling, psamp.extent / 2. + 5 * psamp.sampling)
    H, W = (int(v) for v in osamp.shape)
    thick = numpy.full(S, 15.0, dtype=dtype) if S > 1 else numpy.array([], dtype=dtype)
    phase = rng.normal(0, 0.25, (S, H, W))
    true_obj = (numpy.exp(1j * phase) * rng.uniform(0.9, 1.0, (S, H, W))).astype(cdt)
    est_obj = (numpy.exp(1j * 0.5 * phase) * 0.98).astype(cdt)
    tilts = (rng.normal(0, 2.0, scan.shape).astype(dtype) if tilt else None)

    def state(obj, pr):
        return ReconsState(iter=IterState(0, 0, 0), wavelength=wavelength,
                           probe=ProbeState(psamp, pr.copy()),
                           object=ObjectState(osamp, obj.copy(), thick.copy()),
                           scan=scan.copy(), tilt=None if tilts is None else tilts.copy(),
                           progress=ProgressState.empty())

    # simulate patterns with the reference forward model (gradient-engine form)
    st = state(true_obj, probe * 1.3)
    props = make_propagators(st, 2 / 3)
    flat = numpy.indices(scan.shape[:-1]).reshape(2, -1)
    psi, gobj, _ = cutout_group(ky, kx, st, flat)
    tprops = tilt_propagators(ky, kx, st, props, None if tilts is None else tilts[tuple(flat)])
    def step_fn(i, prop, p):
        if prop is not None:
            return ifft2(fft2(p * gobj[:, i, None]) * prop[:, None])
        return p * gobj[:, i, None]
    wave = fft2(slice_forwards(tprops, psi, step_fn))
    inten = numpy.sum(numpy.abs(wave) ** 2, axis=1)
    pats = rng.poisson(inten * 2e4).astype(dtype) / dtype(2e4)
    pats = pats.reshape(*scan.shape[:-1], N, N)
    mask = numpy.ones((N, N), dtype=dtype)
    mask[0, 0] = 0.5
    return dict(state=state, est_obj=est_obj, probe=probe, scan=scan, pats=pats, mask=mask,
                psamp=psamp, osamp=osamp, thick=thick, tilts=tilts, wavelength=wavelength,
                ky=ky, kx=kx)


def case_arrays(c):
    return dict(probe=c['probe'], object=c['est_obj'], scan=c['scan'], patterns=c['pats'],
                mask=c['mask'], probe_sampling=numpy.asarray(c['psamp'].sampling),
                corner=numpy.asarray(c['osamp'].corner), obj_sampling=numpy.asarray(c['osamp'].sampling),
                thicknesses=c['thick'], wavelength=numpy.float64(c['wavelength']),
                tilt=c['tilts'] if c['tilts'] is not None else numpy.zeros(0, F32))


def group_cases():
    configs = [
        ('lsqml_ms', dict(seed=1, N=32, M=2, S=3, scan_shape=(4, 4), step=2.0), 'lsqml', dict()),
        ('lsqml_ss', dict(seed=2, N=32, M=1, S=1, scan_shape=(3, 4), step=1.6), 'lsqml', dict()),
        ('lsqml_tilt', dict(seed=3, N=32, M=2, S=2, scan_shape=(3, 3), step=2.0, tilt=True), 'lsqml', dict()),
        ('lsqml_noprobe', dict(seed=4, N=32, M=3, S=2, scan_shape=(3, 3), step=2.0), 'lsqml',
         dict(update_probe=False, noise='anscombe')),
        ('lsqml_f64', dict(seed=5, N=32, M=2, S=2, scan_shape=(3, 3), step=2.0, dtype=numpy.float64), 'lsqml', dict()),
        ('epie_ms', dict(seed=6, N=32, M=2, S=3, scan_shape=(4, 4), step=2.0), 'epie', dict()),
        ('epie_ss', dict(seed=7, N=32, M=1, S=1, scan_shape=(3, 4), step=1.6), 'epie', dict(update_object=False)),
    ]
    for name, kw, solver, opts in configs:
        c = make_case(**kw)
        dtype = kw.get('dtype', F32)
        noise_kind = opts.get('noise', 'amplitude')
        nm = (AnscombeNoiseModel(None, AnscombeNoisePlan()) if noise_kind == 'anscombe'
              else AmplitudeNoiseModel(None, AmplitudeNoisePlan(eps=1e-3)))
        st = c['state'](c['est_obj'], c['probe'])
        sim = SimulationState(state=st, noise_model=nm, group_constraints=(), iter_constraints=(),
                              xp=numpy, dtype=dtype)
        props = make_propagators(st, 2 / 3)
        rng = numpy.random.default_rng(100 + kw['seed'])
        n = int(numpy.prod(c['scan'].shape[:-1]))
        pick = rng.permutation(n)[: max(2, (2 * n) // 3)]
        group = numpy.stack(numpy.unravel_index(pick, c['scan'].shape[:-1]))
        gp = c['pats'][tuple(group)]
        flags = dict(update_object=opts.get('update_object', True),
                     update_probe=opts.get('update_probe', True),
                     update_position=True, calc_error=True)
        out = dict(case_arrays(c), group=pick.astype(numpy.int64))
        if solver == 'lsqml':
            plan = LSQMLSolverPlan(beta_object=0.9, beta_probe=0.8, illum_reg_object=1e-2,
                                   illum_reg_probe=1e-2, gamma=1e-4)
            z_o = numpy.zeros(c['probe'].shape[-2:], dtype=dtype)
            z_p = numpy.zeros(c['est_obj'].shape, dtype=dtype)
            om, pm, resc = solvers.lsqml_dry_run(sim, group, gp, pattern_mask=c['mask'], props=props,
                                                 obj_mag=z_o.copy(), probe_mag=z_p.copy())
            sim, nom, npm, errs, pos = solvers.lsqml_run(
                sim, group, gp, pattern_mask=c['mask'], props=props, obj_mag=om, probe_mag=pm,
                new_obj_mag=z_o.copy(), new_probe_mag=z_p.copy(), beta_object=plan.beta_object,
                beta_probe=plan.beta_probe, illum_reg_object=plan.illum_reg_object,
                illum_reg_probe=plan.illum_reg_probe, gamma=plan.gamma, **flags)
            out.update(dry_obj_mag=om, dry_probe_mag=pm, dry_rescale=resc,
                       new_obj_mag=nom, new_probe_mag=npm,
                       params=numpy.array([plan.beta_object, plan.beta_probe, plan.illum_reg_object,
                                           plan.illum_reg_probe, plan.gamma]))
        else:
            plan = EPIESolverPlan(beta_object=0.7, beta_probe=0.6)
            resc = solvers.epie_dry_run(sim, group, gp, pattern_mask=c['mask'], props=props)
            sim, errs, pos = solvers.epie_run(
                sim, group, gp, pattern_mask=c['mask'], props=props, beta_object=plan.beta_object,
                beta_probe=plan.beta_probe, **flags)
            out.update(dry_rescale=resc, params=numpy.array([plan.beta_object, plan.beta_probe]))
        out.update(out_object=sim.state.object.data, out_probe=sim.state.probe.data,
                   errors=errs, pos_update=pos,
                   flags=numpy.array([flags['update_object'], flags['update_probe']]),
                   noise=numpy.array(noise_kind))
        save(f'group_{name}.npz', **out)


def engine_cases():
    for name, solver in (('lsqml', 'lsqml'), ('epie', 'epie')):
        c = make_case(seed=11 if solver == 'lsqml' else 12, N=32, M=2, S=2, scan_shape=(5, 5), step=2.0)
        st = c['state'](c['est_obj'], c['probe'])
        if solver == 'lsqml':
            sol = ConventionalSolverHook('phaser.engines.conventional.solvers:LSQMLSolver',
                                         LSQMLSolverPlan(beta_object=0.9, beta_probe=0.9, gamma=1e-3), 'lsqml')
        else:
            sol = ConventionalSolverHook('phaser.engines.conventional.solvers:EPIESolver',
                                         EPIESolverPlan(beta_object=0.8, beta_probe=0.7), 'epie')
        plan = ConventionalEnginePlan(
            noise_model=NoiseModelHook('phaser.engines.common.noise_models:AmplitudeNoiseModel',
                                       AmplitudeNoisePlan(eps=1e-2), 'amplitude'),
            solver=sol,
            position_solver=PositionSolverHook('phaser.engines.common.position_correction:MomentumPositionSolver',
                                               MomentumPositionSolverProps(step_size=1e-2, max_step_size=0.2,
                                                                           momentum=0.9), 'momentum'),
            group_constraints=[], iter_constraints=[], niter=3, grouping=10,
            update_positions=True, calc_error_fraction=0.5,
        )
        res = run_engine({'data': Patterns(c['pats'].copy(), c['mask'].copy()), 'state': st,
                          'dtype': F32, 'xp': numpy, 'recons_name': 'golden', 'seed': 'golden-seed'}, plan)
        save(f'engine_{name}.npz', **case_arrays(c), out_object=res.object.data, out_probe=res.probe.data,
             out_scan=res.scan, errors=numpy.asarray(res.progress.detector_errors),
             niter=numpy.int64(3), grouping=numpy.int64(10))


def cutout_case():
    rng = numpy.random.default_rng(21)
    samp = ObjectSampling((60, 70), (0.5, 0.75))
    obj = (rng.normal(size=(2, 60, 70)) + 1j * rng.normal(size=(2, 60, 70))).astype(C64)
    # positions include exact half-pixel offsets to pin round-half-to-even
    pos = numpy.array([[0., 0.], [-3.0, 4.5], [2.25, -5.625], [-4.75, -7.875], [5.0, 9.0],
                       [0.125, 0.1875], [-2.5, 2.625]], dtype=F32)
    shape = (16, 12)
    cut = samp.cutout(obj, pos, shape)
    views = (rng.normal(size=(len(pos), 2, *shape)) + 1j * rng.normal(size=(len(pos), 2, *shape))).astype(C64)
    added = samp.add_view_at_pos(obj.copy(), pos, views)
    idx = samp._pos_to_object_idx(pos, shape)
    save('cutouts.npz', obj=obj, pos=pos, shape=numpy.array(shape), corner=samp.corner,
         sampling=samp.sampling, starts=numpy.asarray(cut._start_idxs), idx=idx,
         gathered=cut.get(), views=views, added=added, subpx=samp.get_subpx_shifts(pos, shape))


def numerics_case():
    rng = numpy.random.default_rng(31)
    a8 = (rng.normal(size=(3, 8, 8)) + 1j * rng.normal(size=(3, 8, 8))).astype(C64)
    a5 = (rng.normal(size=(2, 5, 5)) + 1j * rng.normal(size=(2, 5, 5))).astype(C64)
    psamp = Sampling((32, 32), sampling=(0.37, 0.41))
    ky, kx = psamp.recip_grid(dtype=F32, xp=numpy)
    lam = physics.Electron(300e3).wavelength
    probe = optics.make_focused_probe(ky, kx, lam, 25., defocus=200.)
    modes = optics.make_hermetian_modes(probe, 4, 0.7, [0.5, 1/3, 1/6])
    prop = optics.fresnel_propagator(ky, kx, lam, 20., tilt=(3., -2.))
    shifts = rng.uniform(-0.3, 0.3, (4, 2))
    filt = optics.fourier_shift_filter(ky, kx, shifts)
    st = ReconsState(iter=IterState(0, 0, 0), wavelength=lam, probe=ProbeState(psamp, modes),
                     object=ObjectState(ObjectSampling((40, 40), psamp.sampling),
                                        numpy.ones((4, 40, 40), C64), numpy.array([20., 20., 12., 20.], F32)),
                     scan=numpy.zeros((1, 2), F32), progress=ProgressState.empty())
    props = make_propagators(st, 2 / 3)
    raster = scan_mod.make_raster_scan((4, 5), (1.5, 2.0), dtype=F32, xp=numpy)
    save('numerics.npz', a8=a8, a5=a5, fft_a8=fft2(a8), ifft_a8=ifft2(a8), fft_a5=fft2(a5), ifft_a5=ifft2(a5),
         psamp=numpy.asarray(psamp.sampling), wavelength=numpy.float64(lam), probe=probe, modes=modes,
         prop=prop, shifts=shifts, filt=filt, props=props, thick=numpy.array([20., 20., 12., 20.], F32),
         raster=raster)
    # loss values of the three noise models on one set of arrays
    I = rng.uniform(0, 3, (4, 32, 32)).astype(F32)
    P = rng.poisson(I).astype(F32)
    P[0, 0, 0] = -1.0
    m = numpy.ones((32, 32), F32)
    losses = [float(AmplitudeNoiseModel(None, AmplitudeNoisePlan()).calc_loss(None, I, P, m, None)[0]),
              float(AnscombeNoiseModel(None, AnscombeNoisePlan()).calc_loss(None, I, P, m, None)[0]),
              float(PoissonNoiseModel(None, PoissonNoisePlan()).calc_loss(None, I, P, m, None)[0])]
    save('noise_losses.npz', intensity=I, patterns=P, mask=m, losses=numpy.array(losses))


def grouping_case():
    out = {
        'sparse_32_8': [a.tolist() for a in misc.create_sparse_groupings(32, 8, 'seed1')],
        'sparse_33_8': [a.tolist() for a in misc.create_sparse_groupings(33, 8, 'seed1')],
        'sparse_6x7_10_i3': [a.tolist() for a in misc.create_sparse_groupings((6, 7), 10, 'abc', i=3)],
        'shuffle_5_i2': [int(v) for v in misc.shuffled(list(range(5)), seed='abc', i=2)],
        'mask_17_0.1': misc.mask_fraction_of_groups(17, 0.1).tolist(),
        'mask_3_0.5': misc.mask_fraction_of_groups(3, 0.5).tolist(),
        'wavelength_200kV': physics.Electron(200e3).wavelength,
        'wavelength_300kV': physics.Electron(300e3).wavelength,
    }
    scan = numpy.stack(numpy.meshgrid(numpy.linspace(0., 20., 8), numpy.linspace(0., 20., 8),
                                      indexing='ij'), axis=-1).reshape(-1, 2)
    out['compact_64_16'] = [a.tolist() for a in misc.create_compact_groupings(scan, 16, 'seed1')]
    path = HERE / 'groupings.json'
    path.write_text(json.dumps(out, indent=1))
    print(f"wrote {path.name}")


def constraints_case():
    """Iteration constraints and gradient-engine cost regularisers of
    phaser/engines/common/regularizers.py on one small multislice state with
    odd object sides (arbitrary-size DFT filters)."""
    from phaser.engines.common import regularizers as R
    from phaser.hooks.regularization import (RegularizeLayersProps, ObjLowPassProps, GaussianProps,
                                             ClampObjectAmplitudeProps, LimitProbeSupportProps,
                                             CostRegularizerProps, TVRegularizerProps)
    # RegularizeLayers passes the object ARRAY to to_real_dtype
    # (regularizers.py:97), which numpy 2 rejects; cupy and jax arrays go through
    # numpy.dtype's `.dtype` attribute path.  Emulate that path here.
    orig = R.to_real_dtype
    R.to_real_dtype = lambda v: orig(v.dtype if isinstance(v, numpy.ndarray) else v)
    c = make_case(seed=41, N=32, M=2, S=3, scan_shape=(3, 4), step=3.0, samp=0.5)
    rng = numpy.random.default_rng(42)
    S, H, W = c['est_obj'].shape
    obj = (numpy.exp(1j * rng.normal(0, 0.6, (S, H, W))) * rng.uniform(0.7, 1.3, (S, H, W))).astype(C64)
    thick = numpy.array([18., 18., 18.], F32)

    def st():
        s_ = c['state'](obj, c['probe'])
        s_.object.thicknesses = thick.copy()
        return s_

    out = dict(obj=obj, probe=c['probe'], thick=thick, obj_sampling=numpy.asarray(c['osamp'].sampling),
               corner=numpy.asarray(c['osamp'].corner), region_min=numpy.asarray(c['osamp'].region_min),
               region_max=numpy.asarray(c['osamp'].region_max), probe_sampling=numpy.asarray(c['psamp'].sampling),
               wavelength=numpy.float64(c['wavelength']), scan=c['scan'])

    def apply(hook, name, what='object'):
        s_ = st()
        state = hook.init_state(s_)
        s_, _ = hook.apply_iter(s_, state)
        out[name] = numpy.asarray(getattr(s_, what).data)

    apply(R.RegularizeLayers(None, RegularizeLayersProps(sigma=30.0, weight=0.6)), 'layers')
    apply(R.ObjLowPass(None, ObjLowPassProps(max_freq=0.3)), 'low_pass')
    apply(R.ObjGaussian(None, GaussianProps(sigma=0.7, weight=0.8)), 'gaussian')
    apply(R.RemovePhaseRamp(None, {}), 'phase_ramp')
    apply(R.ClampObjectAmplitude(None, ClampObjectAmplitudeProps(amplitude=1.1)), 'clamp')
    apply(R.LimitProbeSupport(None, LimitProbeSupportProps(max_angle=20.0)), 'probe_support', 'probe')
    # tilt_gaussian: nearest-position image of the tilts, Gaussian blur, sampled back
    from phaser.hooks.regularization import TiltGaussianProps
    tilts = rng.normal(0, 2.0, c['scan'].shape).astype(F32)
    s_ = st()

    class _Values(numpy.ndarray):
        # UnstructuredGaussian reads `getattr(values, 'data', values)` (regularizers.py:470),
        # which for a numpy array is its memoryview; jax arrays have no `.data`.  Emulate that.
        @property
        def data(self):
            return numpy.asarray(self)

    s_.tilt = tilts.copy().view(_Values)
    hook = R.UnstructuredGaussian(None, TiltGaussianProps(sigma=0.8, weight=0.7))
    s_, _ = hook.apply_iter(s_, hook.init_state(s_))
    out['tilt_in'] = tilts
    out['tilt_gaussian'] = numpy.asarray(s_.tilt)

    group = numpy.indices((3, 4)).reshape(2, -1)[:, :7]
    costs = {}
    for name, hook in [('obj_l1', R.ObjL1(None, CostRegularizerProps(cost=0.3))),
                       ('obj_l2', R.ObjL2(None, CostRegularizerProps(cost=0.4))),
                       ('obj_phase_l1', R.ObjPhaseL1(None, CostRegularizerProps(cost=0.5))),
                       ('obj_recip_l1', R.ObjRecipL1(None, CostRegularizerProps(cost=0.01))),
                       ('obj_tv', R.ObjTotalVariation(None, TVRegularizerProps(cost=0.6, eps=1e-6))),
                       ('obj_tikh', R.ObjTikhonov(None, CostRegularizerProps(cost=0.7))),
                       ('layers_tv', R.LayersTotalVariation(None, CostRegularizerProps(cost=0.8))),
                       ('layers_tikh', R.LayersTikhonov(None, CostRegularizerProps(cost=0.9))),
                       ('probe_phase_tikh', R.ProbePhaseTikhonov(None, CostRegularizerProps(cost=0.02))),
                       ('probe_recip_tikh', R.ProbeRecipTikhonov(None, CostRegularizerProps(cost=0.03))),
                       ('probe_recip_tv', R.ProbeRecipTotalVariation(None, TVRegularizerProps(cost=0.04)))]:
        s_ = st()
        costs[name] = float(hook.calc_loss_group(group, s_, hook.init_state(s_))[0])
    out['cost_names'] = numpy.array(list(costs))
    out['cost_values'] = numpy.array(list(costs.values()))
    out['cost_group_size'] = numpy.int64(group.shape[-1])
    save('constraints.npz', **out)


def prepare_case():
    """phaser.execute.prepare_for_engine (execute.py:334-402) on one small state under
    several engine plans: detector/probe resizing (pad_crop and resample, up and
    down), object resampling to the probe's pixel size and padding to the scan,
    probe-mode truncation and creation, and z reslicing (multi->multi with each
    alignment's default, single->multi, multi->single)."""
    from phaser.execute import prepare_for_engine
    from phaser.types import SliceList, SliceStep, SliceTotal
    from phaser.utils.object import resample_slices
    c = make_case(seed=31, N=32, M=2, S=3, scan_shape=(4, 4), step=2.0)
    plans = {
        'pad_crop_up': dict(sim_shape=(40, 40), resize_method='pad_crop', probe_modes=2),
        'pad_crop_down': dict(sim_shape=(24, 24), resize_method='pad_crop', probe_modes=2),
        'resample_up': dict(sim_shape=(36, 36), resize_method='resample', probe_modes=2),
        'resample_down': dict(sim_shape=(28, 28), resize_method='resample', probe_modes=2, obj_pad_px=9.0),
        'modes_down': dict(probe_modes=1),
        'modes_up': dict(probe_modes=4, base_mode_power=0.6),
        'reslice': dict(probe_modes=2, slices=SliceStep(n=5, slice_thickness=10.0)),
        'reslice_total': dict(probe_modes=2, slices=SliceTotal(n=2, total_thickness=40.0)),
        'to_single': dict(probe_modes=2, slices=SliceList(thicknesses=[])),
    }
    out = dict(case_arrays(c), osamp_shape=numpy.asarray(c['osamp'].shape),
               region_min=numpy.asarray(c['osamp'].region_min), region_max=numpy.asarray(c['osamp'].region_max))
    names = []
    for name, kw in plans.items():
        st = c['state'](c['est_obj'], c['probe'])
        plan = ConventionalEnginePlan(
            noise_model=NoiseModelHook('phaser.engines.common.noise_models:AmplitudeNoiseModel',
                                       AmplitudeNoisePlan(), 'amplitude'),
            solver=ConventionalSolverHook('phaser.engines.conventional.solvers:LSQMLSolver', LSQMLSolverPlan(),
                                          'lsqml'),
            group_constraints=[], iter_constraints=[], **kw)
        pats, st2 = prepare_for_engine(Patterns(c['pats'].copy(), c['mask'].copy()), st, numpy, plan)
        names.append(name)
        os2 = st2.object.sampling
        out.update({f'{name}__probe': st2.probe.data, f'{name}__probe_sampling': numpy.asarray(st2.probe.sampling.sampling),
                    f'{name}__obj_shape': numpy.asarray(os2.shape),
                    f'{name}__obj_sampling': numpy.asarray(os2.sampling), f'{name}__corner': numpy.asarray(os2.corner),
                    f'{name}__region_min': numpy.asarray(os2.region_min), f'{name}__region_max': numpy.asarray(os2.region_max),
                    f'{name}__thicknesses': numpy.asarray(st2.object.thicknesses)})
        if st2.object.data.shape != c['est_obj'].shape or not numpy.array_equal(st2.object.data, c['est_obj']):
            out[f'{name}__object'] = st2.object.data
        if 'sim_shape' in kw:   # the other plans leave the patterns untouched
            out.update({f'{name}__patterns': pats.patterns, f'{name}__mask': pats.pattern_mask})
        else:
            assert pats.patterns.shape == c['pats'].shape and numpy.array_equal(pats.patterns, c['pats'])
    # resample_slices' other alignment and padding modes, on the same object
    obj = c['est_obj'][:, 20:32, 24:36]
    for align in ('top', 'middle', 'bottom'):
        for pad in ('vacuum', 'edge', 'average'):
            key = f'slices_{align}_{pad}'
            out[key] = resample_slices(obj, c['thick'], [12.0, 9.0, 14.0, 11.0], align=align, pad_mode=pad)
    out['plan_names'] = numpy.array(names)
    save('prepare.npz', **out)


CASES = {'numerics': numerics_case, 'cutouts': cutout_case, 'groupings': grouping_case,
         'groups': group_cases, 'engines': engine_cases, 'constraints': constraints_case,
         'prepare': prepare_case}

if __name__ == '__main__':
    for name in (sys.argv[1:] or list(CASES)):
        CASES[name]()
