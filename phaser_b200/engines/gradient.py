"""Gradient engine on the B200 kernels.

Drop-in for `phaser.engines.gradient.run:run_engine`
(phaser/engines/gradient/run.py:156-349).  The reference differentiates its
forward model with jax; here the fused kernel evaluates the loss and its
hand-written adjoint in one launch per mini-batch (phb_solver_group with
PHB_SOLVER_GRAD), and the optax solvers of phaser/engines/gradient/solvers.py
run as device kernels (phb_optimizer_update).  Structure per iteration, as in
the reference:

  per group   loss + gradients -> descent directions -g / B (probe) and
              -g / (B sum|P|^2) (object, positions) -> every per-group solver
              (object / probe) updates its variables -> group constraints
  per iter    mean loss; per-iteration solvers (positions) from the gathered
              group directions, update minus its mean; iteration constraints;
              positions checked against the object.

Every cost regulariser of the reference (object: obj_l1, obj_l2, obj_phase_l1,
obj_recip_l1, obj_tv, obj_tikh, layers_tv, layers_tikh; probe: probe_phase_tikh,
probe_recip_tikh, probe_recip_tv) adds its value to each group's loss and its
gradient to the object / probe gradient.  Tilts (per position, mrad) are
per-iteration variables like positions: their gradient comes from the fused
kernel's adjoint through the tilted propagators, and their update is added
without removing its mean (run.py:119-123).
"""
from __future__ import annotations

import ctypes
import logging
import typing as t

import numpy
import torch

from .. import plan as P
from .. import _lib
from ..constraints import build_constraints
from ..device import DeviceEngine, _is_complex64
from ..groups import GroupManager
from .conventional import _call, _noise, _object_sampling

logger = logging.getLogger(__name__)

_PER_ITER_VARS = frozenset({'positions', 'tilt'})
_KINDS = {'sgd': _lib.PHB_OPTIM_SGD, 'adam': _lib.PHB_OPTIM_ADAM, 'polyak_sgd': _lib.PHB_OPTIM_POLYAK}



def _array(a):
    """A state array as given: a device tensor stays one, anything else becomes numpy."""
    return a if torch.is_tensor(a) else numpy.asarray(a)


def _host(a) -> numpy.ndarray:
    return a.detach().cpu().numpy() if torch.is_tensor(a) else numpy.asarray(a)

def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _floats(x: torch.Tensor) -> torch.Tensor:
    return torch.view_as_real(x) if x.is_complex() else x


class DeviceSolver:
    """One gradient solver (phaser/engines/gradient/solvers.py:48-138) with its
    optax state on the device.  `params` maps each variable to the device tensor
    it updates in place (positions: the update is written to a scratch tensor and
    added minus its mean, run.py:115-118)."""

    def __init__(self, kind: str, props: t.Any, params: t.Mapping[str, torch.Tensor]):
        self.kind, self.props = kind, props
        self.params = frozenset(params)
        self.count = 0
        self.hyper: t.Dict[str, float] = {}
        if kind == 'sgd':
            self._sched = {'learning_rate': P.get(props, 'learning_rate')}
            if P.get(props, 'momentum', None) is not None:
                self._sched['momentum'] = P.get(props, 'momentum')
        elif kind == 'adam':
            self._sched = {'learning_rate': P.get(props, 'learning_rate')}
        else:
            self._sched = {'max_learning_rate': P.get(props, 'max_learning_rate'),
                           'scaling': P.get(props, 'scaling', 1.0)}
        self._sched = {k: P.process_schedule(v) for (k, v) in self._sched.items()}
        self.state1 = {k: torch.zeros_like(v) for (k, v) in params.items()
                       if kind == 'adam' or (kind == 'sgd' and 'momentum' in self._sched)}
        self.state2 = {k: torch.zeros(v.shape, dtype=torch.float32, device=v.device) for (k, v) in params.items()
                       if kind == 'adam'}
        dev = next(iter(params.values())).device
        self.sq_norm = torch.zeros((1,), dtype=torch.float64, device=dev)

    @classmethod
    def name(cls) -> str:
        return 'gradient'

    def update_for_iter(self, fargs) -> None:
        """Hyper-parameter schedules are evaluated once per iteration (solvers.py:75-80)."""
        self.hyper = {k: f(fargs) for (k, f) in self._sched.items()}

    def update(self, params: t.Mapping[str, torch.Tensor], grads: t.Mapping[str, t.Tuple[torch.Tensor, float]],
               loss: torch.Tensor, *, update_out: t.Optional[t.Mapping[str, torch.Tensor]] = None,
               status: t.Optional[torch.Tensor] = None, status_code: int = 0) -> None:
        """Apply one optax update: grads[k] = (g, scale) with direction d = scale * g.
        `loss` is a device float64 scalar (the Polyak step reads it on the device)."""
        p = self.props
        self.count += 1
        if self.kind == 'polyak_sgd':
            self.sq_norm.zero_()
            for k, (g, scale) in grads.items():
                gf = _floats(g)
                _lib.call('phb_sq_norm_f32', gf.data_ptr(), gf.numel(), float(scale * self.hyper['scaling']),
                          self.sq_norm.data_ptr(), _stream())
        for k, (g, scale) in grads.items():
            o = _lib.PhbOptim()
            o.kind = _KINDS[self.kind]
            o.nesterov = int(bool(P.get(p, 'nesterov', self.kind == 'sgd')))
            prm = params[k]
            out = None if update_out is None else update_out.get(k)
            o.param = 0 if out is not None else prm.data_ptr()
            o.update_out = 0 if out is None else out.data_ptr()
            o.grad = g.data_ptr()
            o.complex_elems = int(prm.is_complex())
            o.n = prm.numel()
            o.grad_scale = float(scale)
            if k in self.state1:
                o.state1 = self.state1[k].data_ptr()
            if k in self.state2:
                o.state2 = self.state2[k].data_ptr()
            o.lr = float(self.hyper.get('learning_rate', 0.0))
            o.momentum = float(self.hyper.get('momentum', 0.0))
            o.b1, o.b2 = float(P.get(p, 'b1', 0.9)), float(P.get(p, 'b2', 0.999))
            o.eps, o.eps_root = float(P.get(p, 'eps', 1e-8)), float(P.get(p, 'eps_root', 0.0))
            o.count = self.count
            if self.kind == 'polyak_sgd':
                o.polyak_sq_norm, o.polyak_loss = self.sq_norm.data_ptr(), loss.data_ptr()
                o.polyak_scaling = float(self.hyper['scaling'])
                o.polyak_max_lr = float(self.hyper['max_learning_rate'])
                o.polyak_f_min = float(P.get(p, 'f_min'))
                o.polyak_eps = float(P.get(p, 'eps', 0.0))
            if status is not None and out is None:
                o.status, o.status_code = status.data_ptr(), int(status_code)
            _lib.call('phb_optimizer_update', ctypes.byref(o), _stream())


_REG_ALIASES = {'obj_tikhonov': 'obj_tikh', 'layers_tikhonov': 'layers_tikh',
                'probe_phase_tikhonov': 'probe_phase_tikh', 'probe_recip_tikhonov': 'probe_recip_tikh'}
_REG_FIELDS = {'obj_l1': 'l1', 'obj_l2': 'l2', 'obj_phase_l1': 'phase_l1', 'obj_tv': 'tv', 'obj_tikh': 'tikh',
               'layers_tv': 'layers_tv', 'layers_tikh': 'layers_tikh'}
_PROBE_FIELDS = {'probe_phase_tikh': 'phase_tikh', 'probe_recip_tikh': 'recip_tikh', 'probe_recip_tv': 'recip_tv'}


class CostRegularizers:
    """The plan's cost regularisers (phaser/engines/common/regularizers.py:195-426),
    evaluated once per group on the device: value into the group loss, gradient
    into the object / probe gradient.  Object terms are scaled by B / n_pos,
    probe terms by 1, as in the reference."""

    def __init__(self, hooks: t.Sequence[t.Any]):
        self.reg = _lib.PhbObjReg()
        self.reg.tv_eps = 1e-8
        self.preg = _lib.PhbProbeReg()
        self.preg.tv_eps = 1e-8
        self.recip_l1 = 0.0
        self.active = self.probe_active = False
        self._scratch: t.Dict[str, torch.Tensor] = {}
        for h in hooks or []:
            if isinstance(h, str):
                name, props = h, {}
            elif isinstance(h, dict):
                h = dict(h)
                name, props = str(h.pop('type')), h
            else:
                name = getattr(h, 'type', None) or getattr(h, 'ref', '')
                props = getattr(h, 'props', None) or {}
                name = P._REF_CLASS_NAMES.get(str(name).rsplit(':', 1)[-1], name)
            name = _REG_ALIASES.get(str(name), str(name))
            cost = float(P.get(props, 'cost'))
            if name in _REG_FIELDS:
                field = _REG_FIELDS[name]
                setattr(self.reg, field, getattr(self.reg, field) + cost)
                if name == 'obj_tv':
                    self.reg.tv_eps = float(P.get(props, 'eps', 1e-8))
                self.active = True
            elif name == 'obj_recip_l1':
                self.recip_l1 += cost
            elif name in _PROBE_FIELDS:
                field = _PROBE_FIELDS[name]
                setattr(self.preg, field, getattr(self.preg, field) + cost)
                if name == 'probe_recip_tv':
                    self.preg.tv_eps = float(P.get(props, 'eps', 1e-8))
                self.probe_active = True
            else:
                raise NotImplementedError(f"cost regularizer '{name}' is not implemented by the B200 backend")

    def _buf(self, key: str, nbytes: int, device) -> torch.Tensor:
        b = self._scratch.get(key)
        if b is None or b.numel() < nbytes:
            b = torch.empty((nbytes,), dtype=torch.uint8, device=device)
            self._scratch[key] = b
        return b

    def apply(self, eng, B: int, grad: t.Optional[torch.Tensor], loss: torch.Tensor,
              grad_probe: t.Optional[torch.Tensor] = None) -> None:
        scale = float(B) / float(eng.n_pos)
        st = _stream()
        if self.active:
            self.reg.scale = scale
            _lib.call('phb_object_regularizers', eng.object.data_ptr(), eng.S, eng.H, eng.W, ctypes.byref(self.reg),
                      0 if grad is None else grad.data_ptr(), loss.data_ptr(), st)
        if self.recip_l1:
            n = eng.lib.phb_object_recip_l1_scratch_bytes(eng.S, eng.H, eng.W)
            buf = self._buf('recip', n, eng.device)
            _lib.call('phb_object_recip_l1', eng.object.data_ptr(), eng.S, eng.H, eng.W, self.recip_l1 * scale,
                      0 if grad is None else grad.data_ptr(), loss.data_ptr(), buf.data_ptr(), st)
        if self.probe_active:
            n = eng.lib.phb_probe_regularizers_scratch_bytes(eng.M, eng.N)
            buf = self._buf('probe', n, eng.device)
            _lib.call('phb_probe_regularizers', eng.probe.data_ptr(), eng.M, eng.N, ctypes.byref(self.preg),
                      0 if grad_probe is None else grad_probe.data_ptr(), loss.data_ptr(), buf.data_ptr(), st)


def process_solvers(props) -> t.Tuple[t.FrozenSet[str], t.List[t.Tuple[t.FrozenSet[str], str, t.Any]],
                                      t.List[t.Tuple[t.FrozenSet[str], str, t.Any]]]:
    """Split the plan's solvers into per-group and per-iteration solvers, with the
    reference's errors for duplicates and mixed sets (run.py:29-65)."""
    seen, duplicate = set(), set()
    group, per_iter = [], []
    solvers = P.get(props, 'solvers', {}) or {}
    for key, hook in dict(solvers).items():
        vs = P.recons_vars(key)
        if not vs:
            continue
        duplicate |= vs & seen
        seen |= vs
        kind, sp = P.gradient_solver(hook)
        if vs <= _PER_ITER_VARS:
            per_iter.append((vs, kind, sp))
            continue
        if vs & _PER_ITER_VARS:
            raise ValueError(f"The same solver can't handle both per-iteration "
                             f"({', '.join(map(repr, sorted(vs & _PER_ITER_VARS)))}) and per-group "
                             f"({', '.join(map(repr, sorted(vs - _PER_ITER_VARS)))}) variables")
        group.append((vs, kind, sp))
    if duplicate:
        raise ValueError(f"Duplicate solvers for variable(s) {', '.join(map(repr, sorted(duplicate)))}.")
    return frozenset(seen), group, per_iter


class GradientEngine:
    """One gradient-engine run on the device: construction uploads the state,
    `presolve()` rescales the probe, `iteration(i)` runs one iteration and
    `finish()` writes the result back into the host state."""

    def __init__(self, args: t.Mapping[str, t.Any], props: t.Any, *,
                 patterns_on_device: t.Optional[torch.Tensor] = None):
        state = args['state']
        data = args['data']
        self.state = state
        self.observer = args.get('observer', None)
        dtype = numpy.dtype(args.get('dtype', numpy.float32))
        if dtype != numpy.float32:
            raise NotImplementedError("the B200 backend computes in float32/complex64 (plan dtype 'float32')")
        self.regularizers = CostRegularizers(P.get(props, 'regularizers', None) or [])
        self.noise = _noise(props)
        self.all_vars, group_specs, iter_specs = process_solvers(props)
        self.niter = int(P.get(props, 'niter', 10))
        self.send_every_group = bool(P.get(props, 'send_every_group', False))
        grouping = int(P.get(props, 'grouping', None) or 64)
        self.compact = bool(P.get(props, 'compact', False))
        self.flags = {
            'probe': P.process_flag(P.get(props, 'update_probe', True)),
            'object': P.process_flag(P.get(props, 'update_object', True)),
            'positions': P.process_flag(P.get(props, 'update_positions', False)),
            'tilt': P.process_flag(P.get(props, 'update_tilt', False)),
        }
        self.shuffle_groups = P.process_flag(P.get(props, 'shuffle_groups', None) or not self.compact)

        probe0 = _array(state.probe.data)
        obj0 = _array(state.object.data)
        self.scan0 = numpy.asarray(state.scan)
        if 'tilt' in self.all_vars and state.tilt is None:
            # a zeroed tilt map, as phaser/execute.py:396-400 creates before the engine runs
            state.tilt = numpy.zeros_like(self.scan0)
        if 'tilt' in self.all_vars and len(numpy.asarray(state.object.thicknesses)) < 2:
            raise ValueError("tilt updates need a multislice object")
        if not (_is_complex64(probe0) and _is_complex64(obj0)):
            raise TypeError("object and probe must be complex64")
        if patterns_on_device is None and torch.is_tensor(data.patterns):
            patterns_on_device = data.patterns   # device-resident patterns (e.g. from prepare_for_engine)
        self.eng = eng = DeviceEngine(
            probe=probe0, obj=obj0, scan=self.scan0,
            patterns=None if patterns_on_device is not None else numpy.asarray(data.patterns),
            mask=_host(data.pattern_mask), probe_sampling=state.probe.sampling.sampling,
            obj_sampling=_object_sampling(state.object.sampling), thicknesses=numpy.asarray(state.object.thicknesses),
            wavelength=float(state.wavelength), tilt=None if state.tilt is None else numpy.asarray(state.tilt),
            noise=self.noise, bwlim_frac=P.get(props, 'bwlim_frac', 2 / 3), group_max=grouping,
            patterns_on_device=patterns_on_device)
        self.params = {'object': eng.object, 'probe': eng.probe, 'positions': eng.scan}
        if 'tilt' in self.all_vars:
            self.params['tilt'] = eng.tilt
        self.group_solvers = [DeviceSolver(k, sp, {v: self.params[v] for v in vs}) for (vs, k, sp) in group_specs]
        self.iter_solvers = [DeviceSolver(k, sp, {v: self.params[v] for v in vs}) for (vs, k, sp) in iter_specs]
        self.group_cons = build_constraints(P.get(props, 'group_constraints', []) or [], eng, state, per_group=True)
        self.iter_cons = build_constraints(P.get(props, 'iter_constraints', []) or [], eng, state, per_group=False)
        self.groups = GroupManager(self.scan0.shape[:-1], grouping, self.compact, seed=args.get('seed', None))

        dev = eng.device
        self.grad_object = torch.zeros_like(eng.object) if 'object' in self.all_vars else None
        self.grad_probe = torch.zeros_like(eng.probe) if 'probe' in self.all_vars else None
        self.grad_pos = torch.zeros_like(eng.scan) if 'positions' in self.all_vars else None
        self.grad_tilt = torch.zeros_like(eng.tilt) if 'tilt' in self.all_vars else None
        self.tilt_step = torch.zeros_like(eng.tilt) if 'tilt' in self.all_vars else None
        self.pos_step = torch.zeros_like(eng.scan)
        self.losses = torch.zeros((len(self.groups),), dtype=torch.float64, device=dev)
        self.loss_mean = torch.zeros((1,), dtype=torch.float64, device=dev)
        # per iteration parity (iteration i reads what iteration i wrote while i + 1 runs):
        # mean loss; status and the count of positions outside the object
        self.loss_hosts = [torch.zeros((2,), dtype=torch.float64).pin_memory() for _ in range(2)]
        self.status_hosts = [torch.zeros((2,), dtype=torch.int32).pin_memory() for _ in range(2)]
        self.probe_int = 0.0
        self.start_i = int(state.iter.total_iter)
        self.fused_events: t.Optional[t.List[t.Tuple[int, int]]] = None
        _call(self.observer, 'init_engine', state, recons_name=args.get('recons_name', ''), plan=props,
              noise_model=self.noise.kind)

    def presolve(self) -> float:
        """Probe intensity rescale over the first groups (run.py:199-212, 413-438)."""
        first = self.groups.iter(self.scan0 if self.compact else None, 0)
        gt, sizes = self.eng.group_tensor([self.groups.flat(g) for g in first])
        rescale = self.eng.presolve(gt, sizes, 'lsqml', gradient_form=True)
        logger.info(f"Rescaling initial probe intensity by {rescale:.2e}")
        self.eng.probe.mul_(float(numpy.sqrt(rescale)))
        self.eng.probe_changed()
        self.probe_int = float(torch.sum(torch.view_as_real(self.eng.probe).double() ** 2))
        if self.observer is not None:   # the reference's state holds the rescaled probe here
            self._refresh_host_state()
        _call(self.observer, 'start_engine', self.state)
        return rescale

    def time_group_steps(self, i: int, warmup: int, steps: int, stream) -> float:
        """Seconds of device time of mini-batches warmup .. warmup + steps - 1 of iteration
        i (loss, adjoint and optimizer steps; not the iteration's tail)."""
        from .conventional import _time_groups
        return _time_groups(self, i, warmup, steps, stream)

    def iteration(self, i: int, *, sync: bool = True, groups_only: t.Optional[int] = None,
                  on_group: t.Optional[t.Callable[[int], None]] = None) -> t.Optional[float]:
        """Run iteration i (1-based).  With sync=True, wait for the device, raise on
        NaN / positions outside the object and return the mean loss.  groups_only=k runs
        only the first k mini-batches (no iteration tail); on_group(gi) is called before
        mini-batch gi is enqueued (timing samples)."""
        eng, state = self.eng, self.state
        state.iter.engine_iter = i
        state.iter.total_iter = self.start_i + i
        fargs = {'state': state, 'niter': self.niter}
        iter_vars = self.all_vars & {k for (k, f) in self.flags.items() if f(fargs)}
        for sol in self.group_solvers + self.iter_solvers:
            sol.update_for_iter(fargs)
        flags = ((_lib.PHB_FLAG_UPDATE_OBJECT if 'object' in iter_vars else 0)
                 | (_lib.PHB_FLAG_UPDATE_PROBE if 'probe' in iter_vars else 0)
                 | (_lib.PHB_FLAG_UPDATE_POSITION if 'positions' in iter_vars else 0)
                 | (_lib.PHB_FLAG_UPDATE_TILT if 'tilt' in iter_vars else 0))
        scan_host = eng.scan.cpu().numpy().reshape(self.scan0.shape) if self.compact else None
        glist = self.groups.iter(scan_host, i, self.shuffle_groups(fargs))
        gt, sizes = eng.group_tensor([self.groups.flat(g) for g in glist])
        if self.losses.numel() < len(sizes):
            self.losses = torch.zeros((len(sizes),), dtype=torch.float64, device=eng.device)
        losses = self.losses[:len(sizes)]
        losses.zero_()
        eng.status.fill_(-1)
        probe_int = self.probe_int
        for gi, B in enumerate(sizes):
            if groups_only is not None and gi >= groups_only:
                return None
            if on_group is not None:
                on_group(gi)
            if 'object' in iter_vars:
                self.grad_object.zero_()
            if 'probe' in iter_vars:
                self.grad_probe.zero_()
            ev = None
            if self.fused_events is not None:
                ev = _new_event_pair()
                self.fused_events.append(ev)
            self._grad_step(gt[gi], B, flags, gi, ev, iter_vars, losses[gi:gi + 1], probe_int)
            self.regularizers.apply(eng, B, self.grad_object if 'object' in iter_vars else None, losses[gi:gi + 1],
                                    self.grad_probe if 'probe' in iter_vars else None)
            dirs = {}
            if 'object' in iter_vars:
                dirs['object'] = (self.grad_object, -1.0 / (probe_int * B))
            if 'probe' in iter_vars:
                dirs['probe'] = (self.grad_probe, -1.0 / B)
            for sol in self.group_solvers:
                d = {k: v for (k, v) in dirs.items() if k in sol.params}
                if d:
                    sol.update(self.params, d, losses[gi:gi + 1], status=eng.status, status_code=gi)
            if 'probe' in iter_vars and any('probe' in s.params for s in self.group_solvers):
                eng.probe_changed()
            for con in self.group_cons:
                con.apply_group()
            if sync and self.observer is not None:
                # run.py:262: after every group, with `force` = send_every_group; a forced
                # update gets the device's current arrays (one wait per group, opted into
                # by the plan), otherwise the state as of the end of the last iteration
                if self.send_every_group:
                    self._refresh_host_state()
                _call(self.observer, 'update_group', state, self.send_every_group)
        torch.mean(losses, dim=0, keepdim=True, out=self.loss_mean)
        for sol in self.iter_solvers:
            d = {}
            if 'positions' in sol.params and 'positions' in iter_vars:
                d['positions'] = (self.grad_pos, 1.0)
            if 'tilt' in sol.params and 'tilt' in iter_vars:
                d['tilt'] = (self.grad_tilt, 1.0)
            if not d:
                continue
            sol.update(self.params, d, self.loss_mean,
                       update_out={'positions': self.pos_step, 'tilt': self.tilt_step})
            if 'positions' in d:
                _lib.call('phb_add_centred', eng.scan.data_ptr(), self.pos_step.data_ptr(), eng.n_pos, _stream())
            if 'tilt' in d:   # the tilt update keeps its mean (run.py:119-123)
                eng.tilt.add_(self.tilt_step)
        for con in self.iter_cons:
            con.apply_iter()
        it_pos = 'positions' in iter_vars
        if it_pos:   # positions outside the object, counted on the device
            eng.count_outside()
        self.loss_hosts[i % 2][:1].copy_(self.loss_mean, non_blocking=True)
        self.status_hosts[i % 2][:1].copy_(eng.status, non_blocking=True)
        if it_pos:
            self.status_hosts[i % 2][1:].copy_(eng.n_outside, non_blocking=True)
        if not sync:
            return None
        torch.cuda.current_stream().synchronize()
        if self.observer is not None:   # observers get the state as it is after iteration i
            self._refresh_host_state()
        return self.check(i, it_pos)

    def _grad_step(self, group: torch.Tensor, B: int, flags: int, gi: int, events, iter_vars, group_loss,
                   probe_int: float) -> None:
        """Loss and gradients of one mini-batch into the engine's gradient buffers."""
        self.eng.step('grad', group, B, flags=flags, group_index=gi, events=events, **self._grad_kw(B, iter_vars,
                                                                                                  group_loss, probe_int))

    def _grad_kw(self, B: int, iter_vars, group_loss, probe_int: float) -> dict:
        return dict(grad_object=self.grad_object if 'object' in iter_vars else None,
                    grad_probe=self.grad_probe if 'probe' in iter_vars else None,
                    grad_pos=self.grad_pos if 'positions' in iter_vars else None,
                    grad_pos_scale=-1.0 / (probe_int * B), group_loss=group_loss,
                    grad_tilt=self.grad_tilt if 'tilt' in iter_vars else None,
                    grad_tilt_scale=-1.0 / (probe_int * B))

    def check(self, i: int, it_pos: bool = True) -> float:
        """Read iteration i's report (after the device has finished iteration i)."""
        state, eng = self.state, self.eng
        rep = self.status_hosts[i % 2]
        bad_group = int(rep[0])
        _lib.raise_for_status(bad_group)
        n_out = int(rep[1])
        if it_pos and n_out > 0:
            raise ValueError(f"{n_out}/{eng.n_pos} probe positions completely outside object")
        loss = float(self.loss_hosts[i % 2][0])
        state.progress.iters = numpy.concatenate([state.progress.iters, [i + self.start_i]])
        state.progress.detector_errors = numpy.concatenate([state.progress.detector_errors, [loss]])
        _call(self.observer, 'update_iteration', state, i, self.niter, loss)
        return loss

    def _refresh_host_state(self) -> None:
        """Copy the device's probe, object, positions and tilt into the host state: the
        one the engine returns and the observers are given.  The reference's state is
        current whenever an observer sees it; SaveObserver writes it out at an iteration
        (observer.py:224-233), the web worker sends it (web/worker.py:79-85)."""
        probe, obj, scan = self.eng.host_state()
        self.state.probe.data = probe
        self.state.object.data = obj
        self.state.scan = scan.astype(self.scan0.dtype)
        if self.eng.tilt is not None and 'tilt' in self.all_vars:
            self.state.tilt = self.eng.tilt.cpu().numpy().reshape(self.scan0.shape).astype(self.scan0.dtype)

    def finish(self):
        self._refresh_host_state()
        _call(self.observer, 'finish_engine', self.state)
        return self.state


def _new_event_pair() -> t.Tuple[int, int]:
    a, b = ctypes.c_void_p(), ctypes.c_void_p()
    _lib.call('phb_event_create', ctypes.byref(a))
    _lib.call('phb_event_create', ctypes.byref(b))
    return a.value, b.value


def run_engine(args: t.Mapping[str, t.Any], props: t.Any) -> t.Any:
    """Run a gradient engine; returns the (updated) ReconsState.
    Signature of phaser.engines.gradient.run:run_engine (run.py:156)."""
    eng = GradientEngine(args, props)
    eng.presolve()
    for i in range(1, eng.niter + 1):
        eng.iteration(i)
    return eng.finish()
