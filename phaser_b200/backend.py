"""Selecting this backend by name from a phaser plan: `backend: b200`.

phaser chooses the array backend of a reconstruction from `ReconsPlan.backend`
(`BackendName`, phaser/types.py:78, resolved by `get_backend_module`,
phaser/utils/num.py:48-68) and the engine of every step from the step's `type`
(`EngineHook.known`, phaser/plan.py:172-173); `execute_plan` / `execute_engine`
(phaser/execute.py:19-85) drive both.  With `backend: b200`, the plan's
`conventional` and `gradient` steps run on this backend's engines, reading the
same plan fields, so an existing plan changes one line:

* between engines the reconstruction state stays in host numpy arrays (the
  backend's array module is numpy); each B200 engine uploads the state, runs
  on the device and writes the result back;
* state preparation before each engine (`prepare_for_engine`,
  phaser/execute.py:334-402) is this backend's device form
  (`phaser_b200.prepare`), after which the state arrays return to the host and
  the patterns stay resident; the reference's "gradient engine requires jax"
  check (execute.py:336-337) does not apply.

`install()` registers the name with an installed phaser at run time, without
editing its sources; a maintainer who prefers a source patch makes the same
four changes (INTEGRATION.md shows them).  `select_engine` is the one decision
the name adds: which function runs an engine step.
"""
from __future__ import annotations

import contextvars
import importlib
import typing as t

import numpy

NAME = 'b200'

# phaser engine type -> this backend's engine (same signature as phaser's run_engine)
ENGINES = {
    'conventional': 'phaser_b200.engines.conventional:run_engine',
    'gradient': 'phaser_b200.engines.gradient:run_engine',
}

# True while execute_plan runs a plan whose backend is b200
_ACTIVE: contextvars.ContextVar[bool] = contextvars.ContextVar('phaser_b200_backend_active', default=False)


def is_b200(backend: t.Any) -> bool:
    return backend is not None and str(backend).lower() == NAME


def engine_function(engine_type: str) -> t.Callable[..., t.Any]:
    """This backend's run_engine for a phaser engine type ('conventional' / 'gradient')."""
    if engine_type not in ENGINES:
        raise NotImplementedError(f"engine type '{engine_type}' has no B200 form "
                                  f"(B200 engines: {', '.join(sorted(ENGINES))})")
    module, fn = ENGINES[engine_type].split(':')
    return getattr(importlib.import_module(module), fn)


def engine_type_of(props: t.Any) -> str:
    """'conventional' or 'gradient' from an engine plan: phaser's ConventionalEnginePlan /
    GradientEnginePlan (or this package's), or a dict that carries a 'type' key."""
    if isinstance(props, dict):
        kind = props.get('type')
        if kind in ENGINES:
            return kind
        if 'solvers' in props:
            return 'gradient'
        if 'solver' in props:
            return 'conventional'
        raise ValueError(f"cannot tell the engine type of plan {sorted(props)}")
    name = type(props).__name__
    if name.startswith('Conventional'):
        return 'conventional'
    if name.startswith('Gradient'):
        return 'gradient'
    raise ValueError(f"cannot tell the engine type of a {name}")


def run_engine(args: t.Mapping[str, t.Any], props: t.Any) -> t.Any:
    """One engine step on this backend, for either engine type (phaser's hook signature)."""
    return engine_function(engine_type_of(props))(args, props)


def select_engine(engine: t.Any, backend: t.Any) -> t.Any:
    """The hook that runs `engine` (a phaser EngineHook: `.props`, called with EngineArgs)
    under `backend`: a B200 engine for 'conventional' / 'gradient' steps when backend is
    b200, else `engine` unchanged."""
    if not is_b200(backend):
        return engine
    props = engine.props
    fn = engine_function(engine_type_of(props))
    return _BoundEngine(fn, props)


class _BoundEngine:
    """A callable with phaser's EngineHook interface (`props`, `__call__(args)`)."""

    def __init__(self, fn: t.Callable[..., t.Any], props: t.Any):
        self.fn = fn
        self.props = props

    def __call__(self, args: t.Mapping[str, t.Any]) -> t.Any:
        return self.fn(args, self.props)

    def __getattr__(self, key: str) -> t.Any:   # plan fields, as phaser's Hook forwards them
        return getattr(self.props, key)


def prepare_for_engine(patterns: t.Any, state: t.Any, engine: t.Any) -> t.Tuple[t.Any, t.Any]:
    """State preparation before a B200 engine: the device form of phaser's
    prepare_for_engine, then the state arrays back to host numpy (observers and
    checkpoints between engines see the reference's array types); the patterns
    stay resident on the device for the engine."""
    import torch
    from . import prepare as PR
    patterns, state = PR.prepare_for_engine(patterns, state, engine)

    def host(a):
        return a.detach().cpu().numpy() if torch.is_tensor(a) else a

    state.probe.data = host(state.probe.data)
    state.object.data = host(state.object.data)
    state.object.thicknesses = host(state.object.thicknesses)
    state.scan = host(state.scan)
    if getattr(state, 'tilt', None) is not None:
        state.tilt = host(state.tilt)
    return patterns, state


def install(phaser_pkg: t.Any = None) -> None:
    """Register `backend: b200` with an installed phaser package (idempotent).

    1. `BackendName` and `ReconsPlan.backend` accept 'b200' (call this before plans
       are parsed);
    2. `get_backend_module('b200')` is numpy (host state between engines);
    3. `execute_plan` records whether the plan's backend is b200;
    4. while it is, `execute_engine` runs `select_engine(...)` and this backend's
       `prepare_for_engine`."""
    if phaser_pkg is None:
        import phaser as phaser_pkg  # noqa: F811
    types = importlib.import_module(phaser_pkg.__name__ + '.types')
    num = importlib.import_module(phaser_pkg.__name__ + '.utils.num')
    execute = importlib.import_module(phaser_pkg.__name__ + '.execute')
    plan = importlib.import_module(phaser_pkg.__name__ + '.plan')
    if getattr(execute, '_b200_installed', False):
        return

    names = tuple(t.get_args(types.BackendName))
    if NAME not in names:
        names = names + (NAME,)
    types.BackendName = t.Literal[names]   # type: ignore[valid-type]
    anns = getattr(plan.ReconsPlan, '__annotations__', {})
    if 'backend' in anns:
        anns['backend'] = t.Optional[t.Literal[names]]   # type: ignore[valid-type]

    orig_backend = num.get_backend_module

    def get_backend_module(backend=None):
        if is_b200(backend):
            return numpy
        return orig_backend(backend)

    num.get_backend_module = get_backend_module
    execute.get_backend_module = get_backend_module

    orig_plan = execute.execute_plan

    def execute_plan(plan_, *args, **kwargs):
        token = _ACTIVE.set(is_b200(getattr(plan_, 'backend', None)))
        try:
            return orig_plan(plan_, *args, **kwargs)
        finally:
            _ACTIVE.reset(token)

    orig_prepare = execute.prepare_for_engine

    def prepare(patterns, state, xp, engine):
        if _ACTIVE.get():
            return prepare_for_engine(patterns, state, engine)
        return orig_prepare(patterns, state, xp, engine)

    orig_engine = execute.execute_engine

    def execute_engine(recons, engine):
        if _ACTIVE.get():
            engine = select_engine(engine, NAME)
        return orig_engine(recons, engine)

    execute.execute_plan = execute_plan
    execute.prepare_for_engine = prepare
    execute.execute_engine = execute_engine
    if getattr(phaser_pkg, 'execute_plan', None) is orig_plan:
        phaser_pkg.execute_plan = execute_plan
    execute._b200_installed = True
