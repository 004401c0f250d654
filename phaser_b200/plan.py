"""Engine plan types for the B200 backend, field-compatible with phaser's.

phaser's own plan classes (phaser/plan.py:43-160, phaser/hooks/solver.py:80-99)
are `pane` dataclasses and its hooks are `Hook(ref, props, type)` objects.
The B200 engines accept those directly (duck-typed), plain dicts of the same
shape (what a plan YAML becomes), or the small dataclasses defined here,
which carry the same field names and defaults.
"""
from __future__ import annotations

import dataclasses
import typing as t


@dataclasses.dataclass(eq=False)
class Flag:
    """Iteration flag (phaser/types.py:125-145): true when after < i, (i-after) % every == 0, i < before."""
    after: int = 0
    every: int = 1
    before: t.Optional[int] = None

    def __call__(self, args) -> bool:
        i = args['state'].iter.engine_iter
        return (self.before is None or i < self.before) and i > self.after and (i - self.after) % self.every == 0


@dataclasses.dataclass(eq=False)
class AmplitudeNoisePlan:
    gaussian_variance: float = 0.1
    eps: float = 1.0e-3
    offset: float = 0.0


@dataclasses.dataclass(eq=False)
class AnscombeNoisePlan(AmplitudeNoisePlan):
    offset: float = 0.375


@dataclasses.dataclass(eq=False)
class PoissonNoisePlan(AmplitudeNoisePlan):
    eps: float = 1.0e-3


@dataclasses.dataclass(eq=False)
class LSQMLSolverPlan:
    stochastic: bool = True
    beta_object: t.Any = 1.0
    beta_probe: t.Any = 1.0
    illum_reg_object: t.Any = 1e-2
    illum_reg_probe: t.Any = 1e-2
    gamma: t.Any = 1e-4


@dataclasses.dataclass(eq=False)
class EPIESolverPlan:
    beta_object: t.Any = 1.0
    beta_probe: t.Any = 1.0


@dataclasses.dataclass(eq=False)
class SteepestDescentPositionSolverProps:
    step_size: float = 1e-2
    max_step_size: t.Optional[float] = None


@dataclasses.dataclass(eq=False)
class MomentumPositionSolverProps:
    step_size: float = 1e-2
    max_step_size: t.Optional[float] = None
    momentum: float = 0.9


@dataclasses.dataclass(eq=False)
class SGDSolverPlan:
    """phaser/plan.py:144-147."""
    learning_rate: t.Any
    momentum: t.Any = None
    nesterov: bool = True


@dataclasses.dataclass(eq=False)
class AdamSolverPlan:
    """phaser/plan.py:150-158."""
    learning_rate: t.Any
    b1: float = 0.9
    b2: float = 0.999
    eps: float = 1.0e-8
    eps_root: float = 0.0
    nesterov: bool = False


@dataclasses.dataclass(eq=False)
class PolyakSGDSolverPlan:
    """phaser/plan.py:161-165."""
    max_learning_rate: t.Any
    f_min: float
    scaling: t.Any = 1.0
    eps: float = 0.0


@dataclasses.dataclass(eq=False)
class HookSpec:
    """A resolved hook: `type` is the registry name ('lsqml', 'amplitude', ...)."""
    type: str
    props: t.Any = None


@dataclasses.dataclass
class SliceList:
    """Slice thicknesses listed (phaser/types.py:95-96)."""
    thicknesses: t.List[float]


@dataclasses.dataclass
class SliceStep:
    """n slices of one thickness (phaser/types.py:98-108)."""
    n: int
    slice_thickness: float

    @property
    def thicknesses(self) -> t.List[float]:
        return [float(self.slice_thickness)] * int(self.n)


@dataclasses.dataclass
class SliceTotal:
    """n equal slices of a total thickness (phaser/types.py:110-120)."""
    n: int
    total_thickness: float

    @property
    def thicknesses(self) -> t.List[float]:
        return [float(self.total_thickness) / int(self.n)] * int(self.n)


def slice_thicknesses(spec: t.Any) -> t.Optional[t.List[float]]:
    """Thicknesses of a `slices` plan entry: a SliceList / SliceStep / SliceTotal (or an
    object with a `thicknesses` attribute), the equivalent dict, a plain list, or None."""
    if spec is None:
        return None
    if isinstance(spec, dict):
        if 'thicknesses' in spec:
            return [float(v) for v in spec['thicknesses']]
        if 'slice_thickness' in spec:
            return SliceStep(int(spec['n']), float(spec['slice_thickness'])).thicknesses
        if 'total_thickness' in spec:
            return SliceTotal(int(spec['n']), float(spec['total_thickness'])).thicknesses
        raise ValueError(f"unknown slices specification {spec!r}")
    if hasattr(spec, 'thicknesses'):
        return [float(v) for v in spec.thicknesses]
    return [float(v) for v in spec]


@dataclasses.dataclass(eq=False)
class ConventionalEnginePlan:
    """Fields of phaser's ConventionalEnginePlan that the engine reads (the EnginePlan
    fields of phaser/plan.py:43-73 included: prepare_for_engine reads sim_shape,
    resize_method, probe_modes, base_mode_power, obj_pad_px and slices)."""
    noise_model: t.Any = dataclasses.field(default_factory=lambda: HookSpec('amplitude', AmplitudeNoisePlan()))
    solver: t.Any = dataclasses.field(default_factory=lambda: HookSpec('lsqml', LSQMLSolverPlan()))
    position_solver: t.Any = None
    group_constraints: t.List[t.Any] = dataclasses.field(default_factory=list)
    iter_constraints: t.List[t.Any] = dataclasses.field(default_factory=list)
    niter: int = 10
    grouping: t.Optional[int] = None
    compact: bool = False
    shuffle_groups: t.Any = None
    buffer_n_groups: int = 2
    update_probe: t.Any = True
    update_object: t.Any = True
    update_positions: t.Any = False
    update_tilt: t.Any = False
    calc_error: t.Any = dataclasses.field(default_factory=lambda: Flag(every=1))
    calc_error_fraction: float = 0.1
    bwlim_frac: t.Optional[float] = 2 / 3
    send_every_group: bool = False
    sim_shape: t.Optional[t.Tuple[int, int]] = None
    resize_method: str = 'pad_crop'
    probe_modes: int = 1
    base_mode_power: float = 0.7
    obj_pad_px: float = 5.0
    slices: t.Any = None


@dataclasses.dataclass(eq=False)
class GradientEnginePlan:
    """Fields of phaser's GradientEnginePlan (phaser/plan.py:43-73, 135-141) that the engine reads."""
    solvers: t.Dict[t.Any, t.Any] = dataclasses.field(default_factory=dict)
    noise_model: t.Any = dataclasses.field(default_factory=lambda: HookSpec('amplitude', AmplitudeNoisePlan()))
    regularizers: t.List[t.Any] = dataclasses.field(default_factory=list)
    group_constraints: t.List[t.Any] = dataclasses.field(default_factory=list)
    iter_constraints: t.List[t.Any] = dataclasses.field(default_factory=list)
    niter: int = 10
    grouping: t.Optional[int] = None
    compact: bool = False
    shuffle_groups: t.Any = None
    buffer_n_groups: int = 2
    update_probe: t.Any = True
    update_object: t.Any = True
    update_positions: t.Any = False
    update_tilt: t.Any = False
    bwlim_frac: t.Optional[float] = 2 / 3
    send_every_group: bool = False
    sim_shape: t.Optional[t.Tuple[int, int]] = None
    resize_method: str = 'pad_crop'
    probe_modes: int = 1
    base_mode_power: float = 0.7
    obj_pad_px: float = 5.0
    slices: t.Any = None


_NOISE_DEFAULTS = {'amplitude': AmplitudeNoisePlan, 'anscombe': AnscombeNoisePlan, 'poisson': PoissonNoisePlan}
_SOLVER_DEFAULTS = {'lsqml': LSQMLSolverPlan, 'epie': EPIESolverPlan}
_POS_DEFAULTS = {'momentum': MomentumPositionSolverProps, 'steepest_descent': SteepestDescentPositionSolverProps}
_GRAD_SOLVER_DEFAULTS = {'sgd': SGDSolverPlan, 'adam': AdamSolverPlan, 'polyak_sgd': PolyakSGDSolverPlan}
_REF_CLASS_NAMES = {
    'AmplitudeNoiseModel': 'amplitude', 'AnscombeNoiseModel': 'anscombe', 'PoissonNoiseModel': 'poisson',
    'LSQMLSolver': 'lsqml', 'EPIESolver': 'epie',
    'MomentumPositionSolver': 'momentum', 'SteepestDescentPositionSolver': 'steepest_descent',
    'ClampObjectAmplitude': 'clamp_object_amplitude', 'LimitProbeSupport': 'limit_probe_support',
    'SGDSolver': 'sgd', 'AdamSolver': 'adam', 'PolyakSGDSolver': 'polyak_sgd',
    'RegularizeLayers': 'layers', 'ObjLowPass': 'obj_low_pass', 'ObjGaussian': 'obj_gaussian',
    'RemovePhaseRamp': 'remove_phase_ramp', 'UnstructuredGaussian': 'tilt_gaussian',
    'ObjL1': 'obj_l1', 'ObjL2': 'obj_l2', 'ObjPhaseL1': 'obj_phase_l1', 'ObjRecipL1': 'obj_recip_l1',
    'ObjTotalVariation': 'obj_tv', 'ObjTikhonov': 'obj_tikh', 'LayersTotalVariation': 'layers_tv',
    'LayersTikhonov': 'layers_tikh', 'ProbePhaseTikhonov': 'probe_phase_tikh',
    'ProbeRecipTikhonov': 'probe_recip_tikh', 'ProbeRecipTotalVariation': 'probe_recip_tv',
}
RECONS_VARS = ('object', 'probe', 'positions', 'tilt')


def resolve_hook(hook: t.Any, defaults: t.Mapping[str, type]) -> t.Tuple[str, t.Any]:
    """(registry name, props) for a phaser Hook, a dict, a string, or a HookSpec."""
    if hook is None:
        raise ValueError("missing hook")
    if isinstance(hook, str):
        name, props = hook, None
    elif isinstance(hook, dict):
        hook = dict(hook)
        name = str(hook.pop('type'))
        props = hook
    else:
        name = getattr(hook, 'type', None) or getattr(hook, 'ref', None)
        props = getattr(hook, 'props', None)
    if name is None:
        raise ValueError(f"can't resolve hook {hook!r}")
    name = str(name)
    if ':' in name:   # 'module:Class' reference to a known reference implementation
        name = _REF_CLASS_NAMES.get(name.rsplit(':', 1)[1], name)
    name = name.lower()
    base = defaults.get(name)
    if base is None:
        raise NotImplementedError(f"hook '{name}' is not implemented by the B200 backend")
    if props is None or props == {}:
        props = base()
    elif isinstance(props, dict):
        props = base(**props)
    return name, props


def noise_model(hook) -> t.Tuple[str, t.Any]:
    return resolve_hook(hook, _NOISE_DEFAULTS)


def solver(hook) -> t.Tuple[str, t.Any]:
    return resolve_hook(hook, _SOLVER_DEFAULTS)


def position_solver(hook) -> t.Optional[t.Tuple[str, t.Any]]:
    return None if hook is None else resolve_hook(hook, _POS_DEFAULTS)


def gradient_solver(hook) -> t.Tuple[str, t.Any]:
    return resolve_hook(hook, _GRAD_SOLVER_DEFAULTS)


def recons_vars(key: t.Any) -> t.FrozenSet[str]:
    """A `solvers` key: a comma-separated string or an iterable of variable
    names (phaser/types.py:280-302)."""
    if isinstance(key, str):
        key = tuple(v.strip() for v in key.split(','))
    out = frozenset(str(v) for v in key)
    bad = out - set(RECONS_VARS)
    if bad:
        raise ValueError(f"unknown reconstruction variable(s) {sorted(bad)}; expected {RECONS_VARS}")
    return out


def process_flag(flag: t.Any) -> t.Callable[[t.Mapping[str, t.Any]], bool]:
    """bool or callable Flag -> predicate of {'state', 'niter'} (phaser/types.py:157-161)."""
    if isinstance(flag, bool) or flag is None:
        val = bool(flag)
        return lambda args: val
    if isinstance(flag, dict):
        flag = Flag(**flag)
    return flag


def process_schedule(sched: t.Any) -> t.Callable[[t.Mapping[str, t.Any]], float]:
    """float, callable, or the plan form of a schedule hook -> value for this
    iteration (phaser/types.py:163-167, phaser/hooks/schedule.py:33-75):
    {'type': 'constant', 'value': v}, {'type': 'piecewise', 'init': s, 'steps':
    {i: s}} (the value of the largest step i <= engine_iter, else init), and
    {'type': 'expr', 'expr': '...'} evaluated with i, iter, state, niter, np."""
    if isinstance(sched, (int, float)):
        val = float(sched)
        return lambda args: val
    if isinstance(sched, dict):
        kind = str(sched.get('type', '')).lower()
        if kind == 'constant':
            return process_schedule(float(sched['value']))
        if kind == 'piecewise':
            init = process_schedule(sched['init'])
            steps = sorted(((int(k), process_schedule(v)) for (k, v) in dict(sched['steps']).items()),
                           key=lambda kv: kv[0], reverse=True)

            def piecewise(args):
                i = args['state'].iter.engine_iter
                for thresh, f in steps:
                    if i >= thresh:
                        return f(args)
                return init(args)
            return piecewise
        if kind == 'expr':
            import numpy
            expr = str(sched['expr'])
            return lambda args: float(eval(expr, {'i': args['state'].iter.engine_iter, 'iter': args['state'].iter,
                                                   'state': args['state'], 'niter': args['niter'], 'np': numpy}))
        raise NotImplementedError(f"schedule type '{kind}' is not implemented by the B200 backend")
    if callable(sched):
        return lambda args: float(sched(args))
    raise TypeError(f"unsupported schedule {sched!r}")


def get(props: t.Any, name: str, default: t.Any = None) -> t.Any:
    if isinstance(props, dict):
        return props.get(name, default)
    return getattr(props, name, default)
