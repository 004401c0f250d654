"""The drop-in boundary on CPU, with the reference's own objects.

The reference phaser package is imported from its sources (through the
test-only `pane` stand-in in tests/golden/pane_shim): its ReconsState,
Patterns, ConventionalEnginePlan and hooks are built exactly as a phaser run
builds them, and passed to this backend

  * through the conventional engine's host adapter, up to the device upload:
    every plan field and state array that reaches the device is the one the
    reference plan and state hold (phaser/engines/conventional/run.py:15-45);
    the upload itself raises without a CUDA device (no CPU fallback);
  * through `backend: b200` selection (phaser_b200.backend.install): the name
    joins BackendName (phaser/types.py:78) and get_backend_module
    (phaser/utils/num.py:48-68), and the reference's own execute_engine
    (phaser/execute.py:47-85) then hands a `conventional` step to this
    backend's engine with the reference's EngineArgs and plan.

Skipped where the reference sources are absent: set PHASER_REF to the phaser
source root (a checkout named `reference` beside this repository is found
without it)."""
import os
import sys

import numpy
import pytest

from .conftest import ROOT


def _reference_root():
    for cand in (os.environ.get('PHASER_REF'), os.path.join(os.path.dirname(ROOT), 'reference')):
        if cand and os.path.isfile(os.path.join(cand, 'phaser', 'execute.py')):
            return cand
    return None


REF = _reference_root()
pytestmark = pytest.mark.skipif(REF is None, reason="phaser reference sources not available (set PHASER_REF)")


@pytest.fixture(scope='module')
def ref():
    # appended, not prepended: the reference tree has its own `tests` package, which must
    # not shadow this repository's (child processes inherit sys.path)
    shim = os.path.join(ROOT, 'tests', 'golden', 'pane_shim')
    added = [p for p in (shim, REF) if p not in sys.path]
    sys.path.extend(added)
    import phaser
    import phaser.execute
    import phaser.plan
    import phaser.state
    import phaser.types
    import phaser.utils.num
    from phaser.hooks import EngineHook
    from phaser.hooks.solver import (NoiseModelHook, ConventionalSolverHook, PositionSolverHook,
                                     MomentumPositionSolverProps)
    from phaser.utils.object import ObjectSampling
    yield dict(phaser=phaser, EngineHook=EngineHook, NoiseModelHook=NoiseModelHook,
               ConventionalSolverHook=ConventionalSolverHook, PositionSolverHook=PositionSolverHook,
               MomentumPositionSolverProps=MomentumPositionSolverProps, ObjectSampling=ObjectSampling)
    for p in added:
        sys.path.remove(p)


def reference_inputs(ref, N=64, M=2, S=3):
    """A reference ReconsState / Patterns / ConventionalEnginePlan of a small reconstruction."""
    from phaser.state import ReconsState, ProbeState, ObjectState, IterState, ProgressState, Patterns
    from phaser.plan import ConventionalEnginePlan, LSQMLSolverPlan, AmplitudeNoisePlan
    from phaser.utils.num import Sampling
    rng = numpy.random.default_rng(5)
    psamp = Sampling((N, N), sampling=(0.2, 0.2))
    scan = (numpy.stack(numpy.meshgrid(numpy.arange(4.), numpy.arange(4.), indexing='ij'), -1) * 0.8
            ).astype(numpy.float32)
    osamp = ref['ObjectSampling'].from_scan(scan, psamp.sampling, psamp.extent / 2. + 5 * psamp.sampling)
    H, W = (int(v) for v in osamp.shape)
    probe = (rng.normal(size=(M, N, N)) + 1j * rng.normal(size=(M, N, N))).astype(numpy.complex64)
    obj = numpy.exp(1j * rng.normal(0, 0.1, (S, H, W))).astype(numpy.complex64)
    thick = numpy.full(S, 20.0, numpy.float32)
    state = ReconsState(iter=IterState(0, 0, 0), wavelength=0.0197, probe=ProbeState(psamp, probe),
                        object=ObjectState(osamp, obj, thick), scan=scan, tilt=None,
                        progress=ProgressState.empty())
    pats = rng.uniform(0, 2, (4, 4, N, N)).astype(numpy.float32)
    mask = numpy.ones((N, N), numpy.float32)
    plan = ConventionalEnginePlan(
        noise_model=ref['NoiseModelHook']('phaser.engines.common.noise_models:AmplitudeNoiseModel',
                                          AmplitudeNoisePlan(eps=1e-2), 'amplitude'),
        solver=ref['ConventionalSolverHook']('phaser.engines.conventional.solvers:LSQMLSolver',
                                             LSQMLSolverPlan(beta_object=0.9, beta_probe=0.8, gamma=1e-3), 'lsqml'),
        position_solver=ref['PositionSolverHook'](
            'phaser.engines.common.position_correction:MomentumPositionSolver',
            ref['MomentumPositionSolverProps'](step_size=1e-2, max_step_size=0.2, momentum=0.9), 'momentum'),
        group_constraints=[], iter_constraints=[], niter=3, grouping=10, update_positions=True,
        calc_error_fraction=0.5)
    return state, Patterns(pats, mask), plan


def test_reference_objects_reach_the_device_upload_unchanged(ref):
    from phaser_b200.engines.conventional import ConventionalEngine, host_inputs
    from phaser_b200.device import NoiseSpec
    state, patterns, plan = reference_inputs(ref)
    args = {'data': patterns, 'state': state, 'dtype': numpy.float32, 'xp': numpy, 'recons_name': 'r',
            'observer': None, 'seed': 'seed'}
    h = host_inputs(args, plan)
    assert h.solver_kind == 'lsqml'
    assert h.noise == NoiseSpec('amplitude', 1e-2, 0.0, 0.1)
    assert h.pos_solver[0] == 'momentum'
    assert h.pos_solver[1].step_size == 1e-2 and h.pos_solver[1].max_step_size == 0.2
    assert (h.niter, h.grouping, h.compact) == (3, 10, False)
    st = {'state': state, 'niter': 3}
    state.iter.engine_iter = 1
    assert h.update_positions(st) and h.update_object(st) and h.update_probe(st) and h.calc_error(st)
    d = h.device_kwargs
    assert d['probe'] is state.probe.data and d['obj'] is state.object.data
    assert numpy.array_equal(d['scan'], state.scan) and numpy.array_equal(d['patterns'], patterns.patterns)
    assert numpy.array_equal(d['mask'], patterns.pattern_mask)
    assert tuple(d['probe_sampling']) == tuple(state.probe.sampling.sampling)
    assert tuple(d['obj_sampling'].corner) == tuple(state.object.sampling.corner)
    assert tuple(d['obj_sampling'].sampling) == tuple(state.object.sampling.sampling)
    assert tuple(d['obj_sampling'].shape) == tuple(state.object.sampling.shape)
    assert numpy.array_equal(d['thicknesses'], state.object.thicknesses)
    assert d['wavelength'] == pytest.approx(0.0197) and d['group_max'] == 10 and d['tilt'] is None
    # the upload: a CUDA device is required, there is no CPU path
    import torch
    if not torch.cuda.is_available():
        with pytest.raises(RuntimeError, match='CUDA device'):
            ConventionalEngine(args, plan)
    # the reference's dtype check (conventional/run.py:42-45)
    with pytest.raises(NotImplementedError):
        host_inputs(dict(args, dtype=numpy.float64), plan)


def test_backend_b200_selects_the_b200_engines(ref, monkeypatch):
    from phaser_b200 import backend
    phaser = ref['phaser']
    backend.install(phaser)
    backend.install(phaser)   # idempotent
    import phaser.execute as ex
    import phaser.plan as pl
    import phaser.types as ty
    import phaser.utils.num as num
    import typing as t
    assert 'b200' in t.get_args(ty.BackendName)
    assert 'b200' in t.get_args(t.get_args(pl.ReconsPlan.__annotations__['backend'])[0])
    assert num.get_backend_module('b200') is numpy and ex.get_backend_module('B200') is numpy
    assert num.get_backend_module('numpy') is numpy

    state, patterns, plan = reference_inputs(ref)
    hook = ref['EngineHook']('phaser.engines.conventional.run:run_engine', plan, 'conventional')
    assert backend.select_engine(hook, 'numpy') is hook
    sel = backend.select_engine(hook, 'b200')
    from phaser_b200.engines.conventional import run_engine as b200_run
    assert sel.fn is b200_run and sel.props is plan and sel.niter == 3

    # the reference's execute_engine, with backend b200 active, calls this backend's engine with
    # the reference's EngineArgs and plan (engine and device preparation stubbed: no GPU here)
    seen = {}

    def engine_stub(args, props):
        seen.update(args=args, props=props)
        return args['state']

    monkeypatch.setitem(backend.ENGINES, 'conventional', 'tests.test_backend_selection:_stub')
    monkeypatch.setattr(sys.modules[__name__], '_stub', engine_stub, raising=False)
    monkeypatch.setattr(backend, 'prepare_for_engine', lambda p, s, e: (p, s))
    from phaser.state import PreparedRecons
    from phaser.observer import ObserverSet
    recons = PreparedRecons(patterns, state, 'r', ObserverSet(()))
    token = backend._ACTIVE.set(True)
    try:
        out = ex.execute_engine(recons, hook)
    finally:
        backend._ACTIVE.reset(token)
    assert seen['props'] is plan
    assert seen['args']['state'] is state and seen['args']['data'] is patterns
    assert set(seen['args']) == {'data', 'state', 'dtype', 'xp', 'recons_name', 'observer', 'seed'}
    assert out.state is state and state.iter.engine_num == 1
    # without backend b200 the reference's own engine hook is used: nothing is redirected
    assert backend.select_engine(hook, None) is hook


def test_engine_type_of_plans(ref):
    from phaser_b200 import backend
    from phaser_b200 import plan as PL
    _, _, plan = reference_inputs(ref)
    assert backend.engine_type_of(plan) == 'conventional'
    assert backend.engine_type_of(PL.GradientEnginePlan(solvers={})) == 'gradient'
    assert backend.engine_type_of({'type': 'gradient'}) == 'gradient'
    assert backend.engine_type_of({'solver': {'type': 'lsqml'}}) == 'conventional'
    with pytest.raises(NotImplementedError):
        backend.engine_function('ptychoshelves')
