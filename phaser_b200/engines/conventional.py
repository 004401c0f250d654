"""Conventional (LSQ-ML / ePIE) engine on the B200 kernels.

Drop-in for `phaser.engines.conventional.run:run_engine`
(phaser/engines/conventional/run.py:15-123): same EngineArgs / plan inputs,
same iteration structure (presolve rescale, per-iteration groupings, group
steps, iteration constraints, position update, detector error), same
exceptions.  Each mini-batch is one fused kernel launch plus small apply
kernels (libphaser_b200, phb_solver_group); the host only builds the seeded
groupings and reads back one status block per iteration.
"""
from __future__ import annotations

import dataclasses
import logging
import typing as t

import numpy
import torch

from .. import plan as P
from .. import _lib
from ..constraints import build_constraints
from ..device import DeviceEngine, NoiseSpec, _is_complex64
from ..groups import GroupManager, mask_fraction_of_groups
from ..sampling import ObjectSampling

logger = logging.getLogger(__name__)



def _array(a):
    """A state array as given: a device tensor stays one, anything else becomes numpy."""
    return a if torch.is_tensor(a) else numpy.asarray(a)


def _host(a) -> numpy.ndarray:
    return a.detach().cpu().numpy() if torch.is_tensor(a) else numpy.asarray(a)

def _object_sampling(s) -> ObjectSampling:
    if isinstance(s, ObjectSampling):
        return s
    return ObjectSampling(tuple(s.shape), s.sampling, s.corner,
                          getattr(s, 'region_min', None), getattr(s, 'region_max', None))


def _noise(props) -> NoiseSpec:
    kind, np_ = P.noise_model(P.get(props, 'noise_model'))
    return NoiseSpec(kind, float(P.get(np_, 'eps', 1e-3)), float(P.get(np_, 'offset', 0.0)),
                     float(P.get(np_, 'gaussian_variance', 0.1)))


def _call(observer, name: str, *args, **kwargs) -> None:
    f = getattr(observer, name, None) if observer is not None else None
    if callable(f):
        f(*args, **kwargs)


class _SolverBase:
    kind = ''

    def __init__(self, engine_plan, props):
        self.engine_plan = engine_plan
        self.plan = props

    @classmethod
    def name(cls) -> str:
        return cls.__name__.replace('Solver', '')

    def schedules(self, fargs) -> t.Dict[str, float]:
        out = {}
        for key, default in (('beta_object', 1.0), ('beta_probe', 1.0), ('illum_reg_object', 1e-2),
                             ('illum_reg_probe', 1e-2), ('gamma', 1e-4)):
            out[key] = P.process_schedule(P.get(self.plan, key, default))(fargs)
        return out


class LSQMLSolver(_SolverBase):
    """LSQ-ML (phaser/engines/conventional/solvers.py:18-128) on the fused kernel."""
    kind = 'lsqml'


class EPIESolver(_SolverBase):
    """ePIE / 3PIE (phaser/engines/conventional/solvers.py:293-383) on the fused kernel."""
    kind = 'epie'


SOLVERS = {'lsqml': LSQMLSolver, 'epie': EPIESolver}


@dataclasses.dataclass
class HostInputs:
    """What the conventional engine reads from EngineArgs and the plan before any
    device work: the parsed plan fields and the exact arguments of the upload."""
    state: t.Any
    observer: t.Any
    noise: NoiseSpec
    solver_kind: str
    solver_props: t.Any
    pos_solver: t.Optional[t.Tuple[str, t.Any]]
    niter: int
    grouping: int
    compact: bool
    update_probe: t.Callable
    update_object: t.Callable
    update_positions: t.Callable
    calc_error: t.Callable
    shuffle_groups: t.Callable
    device_kwargs: t.Dict[str, t.Any]


def host_inputs(args: t.Mapping[str, t.Any], props: t.Any, *,
                patterns_on_device: t.Optional[torch.Tensor] = None) -> HostInputs:
    """Parse EngineArgs (phaser/hooks/__init__.py:174-181) and a conventional engine plan
    (the reference's ConventionalEnginePlan, a dict of the same shape, or
    phaser_b200.plan.ConventionalEnginePlan) on the host, with the reference's checks
    (conventional/run.py:15-45).  No device work happens here."""
    state = args['state']
    data = args['data']
    dtype = numpy.dtype(args.get('dtype', numpy.float32))
    if dtype != numpy.float32:
        raise NotImplementedError("the B200 backend computes in float32/complex64 (plan dtype 'float32')")
    noise = _noise(props)
    if noise.kind == 'poisson':
        # the reference's Poisson model has no wave update (noise_models.py:104-112)
        raise NotImplementedError("the Poisson noise model has no wave update; use 'amplitude' or 'anscombe'")
    solver_kind, solver_props = P.solver(P.get(props, 'solver'))
    compact = bool(P.get(props, 'compact', False))
    probe0 = _array(state.probe.data)
    obj0 = _array(state.object.data)
    scan0 = numpy.asarray(state.scan)
    if not (_is_complex64(probe0) and _is_complex64(obj0)):
        raise TypeError("object and probe must be complex64")
    if patterns_on_device is None and torch.is_tensor(data.patterns):
        patterns_on_device = data.patterns   # device-resident patterns (e.g. from prepare_for_engine)
    grouping = int(P.get(props, 'grouping', None) or 64)
    device_kwargs = dict(
        probe=probe0, obj=obj0, scan=scan0,
        patterns=None if patterns_on_device is not None else numpy.asarray(data.patterns),
        mask=_host(data.pattern_mask), probe_sampling=state.probe.sampling.sampling,
        obj_sampling=_object_sampling(state.object.sampling), thicknesses=numpy.asarray(state.object.thicknesses),
        wavelength=float(state.wavelength), tilt=None if state.tilt is None else numpy.asarray(state.tilt),
        noise=noise, bwlim_frac=P.get(props, 'bwlim_frac', 2 / 3), group_max=grouping,
        patterns_on_device=patterns_on_device)
    return HostInputs(
        state=state, observer=args.get('observer', None), noise=noise, solver_kind=solver_kind,
        solver_props=solver_props, pos_solver=P.position_solver(P.get(props, 'position_solver')),
        niter=int(P.get(props, 'niter', 10)), grouping=grouping, compact=compact,
        update_probe=P.process_flag(P.get(props, 'update_probe', True)),
        update_object=P.process_flag(P.get(props, 'update_object', True)),
        update_positions=P.process_flag(P.get(props, 'update_positions', False)),
        calc_error=P.process_flag(P.get(props, 'calc_error', P.Flag(every=1))),
        shuffle_groups=P.process_flag(P.get(props, 'shuffle_groups', None) or not compact),
        device_kwargs=device_kwargs)


class ConventionalEngine:
    """One conventional-engine run on the device: construction uploads the
    state, `presolve()` rescales the probe, `iteration(i)` runs one full
    iteration (all mini-batches, constraints, position update, error), and
    `finish()` writes the result back into the host state."""

    def __init__(self, args: t.Mapping[str, t.Any], props: t.Any, *,
                 patterns_on_device: t.Optional[torch.Tensor] = None):
        h = host_inputs(args, props, patterns_on_device=patterns_on_device)
        state = self.state = h.state
        self.observer = h.observer
        self.send_every_group = bool(P.get(props, 'send_every_group', False))
        self.noise = h.noise
        self.solver_kind = h.solver_kind
        self.solver = SOLVERS[self.solver_kind](props, h.solver_props)
        self.pos_solver = h.pos_solver
        self.niter = h.niter
        grouping = h.grouping
        self.compact = h.compact
        self.update_probe, self.update_object = h.update_probe, h.update_object
        self.update_positions, self.calc_error = h.update_positions, h.calc_error
        self.shuffle_groups = h.shuffle_groups
        self.scan0 = h.device_kwargs['scan']
        self.eng = eng = DeviceEngine(**h.device_kwargs)   # the upload: raises without a CUDA device
        self.group_cons = build_constraints(P.get(props, 'group_constraints', []) or [], eng, state, per_group=True)
        self.iter_cons = build_constraints(P.get(props, 'iter_constraints', []) or [], eng, state, per_group=False)
        self.groups = GroupManager(self.scan0.shape[:-1], grouping, self.compact, seed=args.get('seed', None))
        self.calc_error_mask = mask_fraction_of_groups(len(self.groups),
                                                       float(P.get(props, 'calc_error_fraction', 0.1)))
        self.mom_state = None
        if self.pos_solver is not None and self.pos_solver[0] == 'momentum':
            self.mom_state = torch.zeros_like(eng.scan)
        self.start_i = int(state.iter.total_iter)
        # two pinned report blocks: iteration i+1 may run while iteration i's report is read
        self.status_hosts = [torch.empty((4,), dtype=torch.float64).pin_memory() for _ in range(2)]
        self.fused_events: t.Optional[t.List[t.Tuple[int, int]]] = None
        _call(self.observer, 'init_engine', state, recons_name=args.get('recons_name', ''), plan=props,
              noise_model=self.noise.kind)

    def presolve(self) -> float:
        """Probe intensity rescale (solvers.py:36-63, 306-329)."""
        first = self.groups.iter(self.scan0 if self.compact else None, 0)
        gt, sizes = self.eng.group_tensor([self.groups.flat(g) for g in first])
        rescale = self.eng.presolve(gt, sizes, self.solver_kind)
        logger.info(f"Rescaling initial probe intensity by {rescale:.2e}")
        self.eng.probe.mul_(float(numpy.sqrt(rescale)))
        self.eng.probe_changed()
        if self.observer is not None:   # the reference's state holds the rescaled probe here
            self._refresh_host_state()
        _call(self.observer, 'start_engine', self.state)
        return rescale

    def time_group_steps(self, i: int, warmup: int, steps: int, stream) -> float:
        """Seconds of device time (CUDA events on `stream`) of mini-batches warmup ..
        warmup + steps - 1 of iteration i, run as the iteration runs them (the iteration's
        tail -- position update, report -- is not part of the sample)."""
        return _time_groups(self, i, warmup, steps, stream)

    def iteration(self, i: int, *, sync: bool = True, groups_only: t.Optional[int] = None,
                  on_group: t.Optional[t.Callable[[int], None]] = None) -> t.Optional[float]:
        """Run iteration i (1-based).  With sync=True, wait for the device, raise
        on NaN / positions outside the object, record and return the error.
        groups_only=k runs only the first k mini-batches (no iteration tail); on_group(gi)
        is called before mini-batch gi is enqueued (timing samples)."""
        eng, state = self.eng, self.state
        state.iter.engine_iter = i
        state.iter.total_iter = self.start_i + i
        fargs = {'state': state, 'niter': self.niter}
        it_pos = self.update_positions(fargs)
        it_err = self.calc_error(fargs)
        flags = ((_lib.PHB_FLAG_UPDATE_OBJECT if self.update_object(fargs) else 0)
                 | (_lib.PHB_FLAG_UPDATE_PROBE if self.update_probe(fargs) else 0)
                 | (_lib.PHB_FLAG_UPDATE_POSITION if it_pos else 0))
        sched = self.solver.schedules(fargs)
        scan_host = eng.scan.cpu().numpy().reshape(self.scan0.shape) if self.compact else None
        glist = self.groups.iter(scan_host, i, self.shuffle_groups(fargs))
        gt, sizes = eng.group_tensor([self.groups.flat(g) for g in glist])
        eng.iteration_reset()
        for gi, B in enumerate(sizes):
            if groups_only is not None and gi >= groups_only:
                return None
            if on_group is not None:
                on_group(gi)
            f = flags | (_lib.PHB_FLAG_CALC_ERROR if (it_err and self.calc_error_mask[gi]) else 0)
            ev = None
            if self.fused_events is not None:
                ev = _new_event_pair()
                self.fused_events.append(ev)
            self._group_step(gt[gi], B, f, gi, ev, sched)
            for con in self.group_cons:
                con.apply_group()
            if sync and self.observer is not None:
                # solvers.py:119, 377: after every group, with `force` = send_every_group; a
                # forced update gets the device's current arrays (one wait per group, opted
                # into by the plan), otherwise the state as of the end of the last iteration
                if self.send_every_group:
                    self._refresh_host_state()
                _call(self.observer, 'update_group', state, self.send_every_group)
        for con in self.iter_cons:
            con.apply_iter()
        if it_pos:
            if self.pos_solver is None:
                raise ValueError("Updating positions with no PositionSolver specified")
            kind, pp = self.pos_solver
            step = float(P.get(pp, 'step_size', 1e-2))
            # the reference's steepest-descent solver clips at step_size (position_correction.py:16)
            maxs = P.get(pp, 'max_step_size', None) if kind == 'momentum' else step
            eng.position_update(self.mom_state, step, maxs, float(P.get(pp, 'momentum', 0.9)))
        # one device->host status block per iteration
        eng.iteration_report(eng.report)
        self._combine_report(eng.report)
        self.status_hosts[i % 2].copy_(eng.report, non_blocking=True)
        if not sync:
            return None
        torch.cuda.current_stream().synchronize()
        if self.observer is not None:   # observers get the state as it is after iteration i
            self._refresh_host_state()
        return self.check(i, it_pos, it_err)

    def _group_step(self, group: torch.Tensor, B: int, flags: int, gi: int, events, sched) -> None:
        """One mini-batch on this device (the data-parallel engine splits it over ranks)."""
        self.eng.step(self.solver_kind, group, B, flags=flags, group_index=gi, events=events, **sched)

    def _combine_report(self, report: torch.Tensor) -> None:
        """Hook for combining the iteration report over ranks (single device: nothing)."""

    def check(self, i: int, it_pos: bool = True, it_err: bool = True) -> t.Optional[float]:
        """Read iteration i's report (after the device has finished iteration i)."""
        state, eng = self.state, self.eng
        rep = self.status_hosts[i % 2]
        bad_group, n_out, err = int(rep[0]), int(rep[1]), float(rep[2])
        _lib.raise_for_status(bad_group)
        if it_pos and n_out > 0:
            raise ValueError(f"{n_out}/{eng.n_pos} probe positions completely outside object")
        error = err if it_err else None
        if error is not None:
            state.progress.iters = numpy.concatenate([state.progress.iters, [i + self.start_i]])
            state.progress.detector_errors = numpy.concatenate([state.progress.detector_errors, [error]])
        _call(self.observer, 'update_iteration', state, i, self.niter, error)
        return error

    def _refresh_host_state(self) -> None:
        """Copy the device's probe, object and positions into the host state: the one the
        engine returns and the observers are given.  The reference's state is current
        whenever an observer sees it; SaveObserver writes it out at an iteration
        (observer.py:224-233), the web worker sends it (web/worker.py:84-85)."""
        probe, obj, scan = self.eng.host_state()
        self.state.probe.data = probe
        self.state.object.data = obj
        self.state.scan = scan.astype(self.scan0.dtype)

    def finish(self):
        self._refresh_host_state()
        _call(self.observer, 'finish_engine', self.state)
        return self.state


def _time_groups(engine, i: int, warmup: int, steps: int, stream) -> float:
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def mark(gi: int) -> None:
        if gi == warmup:
            e0.record(stream)

    engine.iteration(i, sync=False, groups_only=warmup + steps, on_group=mark)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3


def _new_event_pair() -> t.Tuple[int, int]:
    import ctypes
    a, b = ctypes.c_void_p(), ctypes.c_void_p()
    _lib.call('phb_event_create', ctypes.byref(a))
    _lib.call('phb_event_create', ctypes.byref(b))
    return a.value, b.value


def run_engine(args: t.Mapping[str, t.Any], props: t.Any) -> t.Any:
    """Run a conventional engine; returns the (updated) ReconsState.
    Signature of phaser.engines.conventional.run:run_engine (run.py:15)."""
    eng = ConventionalEngine(args, props)
    eng.presolve()
    for i in range(1, eng.niter + 1):
        eng.iteration(i)
    return eng.finish()
