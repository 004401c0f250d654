"""Observers see the state the reference's engines show them (phaser/observer.py):
after every iteration the probe, object and positions as they are after that
iteration (SaveObserver writes them out then, observer.py:224-233), and an
update_group call after every group (conventional/solvers.py:119, 377;
gradient/run.py:262) whose state carries the device's arrays when the plan's
send_every_group forces the update."""
import numpy
import pytest

from phaser_b200 import plan as PL
from phaser_b200.engines.conventional import run_engine as run_conventional
from phaser_b200.engines.gradient import run_engine as run_gradient
from phaser_b200.state import Patterns

from .cases import make_case
from .test_gpu_engine import make_state

pytestmark = pytest.mark.gpu


class Recorder:
    """Keeps copies of what each observer call was shown."""

    def __init__(self):
        self.iters, self.groups, self.start, self.finished = [], [], None, None

    def start_engine(self, state):
        self.start = (state.object.data.copy(), state.probe.data.copy())

    def update_iteration(self, state, i, n, error=None):
        self.iters.append((i, n, state.object.data.copy(), state.probe.data.copy(), numpy.array(state.scan)))

    def update_group(self, state, force=False):
        self.groups.append((force, state.object.data.copy()))

    def finish_engine(self, state):
        self.finished = state.object.data.copy()


def run_args(c, rec, seed):
    return {'data': Patterns(c.patterns, c.mask), 'state': make_state(c), 'dtype': numpy.float32, 'seed': seed,
            'recons_name': 't', 'observer': rec}


def test_conventional_engine_observers_see_every_iteration():
    c = make_case(seed=61, N=64, M=2, S=2, scan_shape=(5, 5))
    props = PL.ConventionalEnginePlan(
        noise_model={'type': 'amplitude', 'eps': 1e-2},
        solver={'type': 'lsqml', 'beta_object': 0.9, 'beta_probe': 0.8, 'gamma': 1e-3},
        position_solver={'type': 'momentum', 'step_size': 1e-2, 'max_step_size': 0.2, 'momentum': 0.9},
        niter=3, grouping=10, update_positions=True, calc_error_fraction=1.0)
    rec = Recorder()
    state = run_conventional(run_args(c, rec, 'observer-seed'), props)
    assert [(i, n) for (i, n, *_) in rec.iters] == [(1, 3), (2, 3), (3, 3)]
    objs = [c.obj] + [r[2] for r in rec.iters]
    for a, b in zip(objs, objs[1:]):   # each iteration's observer saw that iteration's object
        assert not numpy.array_equal(a, b)
    _, _, obj, probe, scan = rec.iters[-1]
    assert numpy.array_equal(obj, state.object.data)
    assert numpy.array_equal(probe, state.probe.data)
    assert numpy.array_equal(scan, state.scan)
    assert numpy.array_equal(rec.finished, state.object.data)
    # one unforced update_group per group, with the state of the last iteration boundary
    n_groups = len(rec.groups) // 3
    assert n_groups >= 2 and len(rec.groups) == 3 * n_groups
    assert all(force is False for (force, _) in rec.groups)
    assert all(numpy.array_equal(o, rec.start[0]) for (_, o) in rec.groups[:n_groups])
    assert all(numpy.array_equal(o, rec.iters[0][2]) for (_, o) in rec.groups[n_groups:2 * n_groups])


@pytest.mark.parametrize('every', [False, True])
def test_gradient_engine_reports_every_group(every):
    c = make_case(seed=62, N=64, M=2, S=2, scan_shape=(5, 5))
    props = PL.GradientEnginePlan(
        solvers={'object': {'type': 'adam', 'learning_rate': 1e-2}, 'probe': {'type': 'adam', 'learning_rate': 1e-3}},
        noise_model={'type': 'amplitude', 'eps': 1e-2}, niter=2, grouping=10, send_every_group=every)
    rec = Recorder()
    state = run_gradient(run_args(c, rec, 'observer-seed'), props)
    assert len(rec.iters) == 2
    n_groups = len(rec.groups) // 2
    assert n_groups >= 2 and len(rec.groups) == 2 * n_groups
    assert all(force == every for (force, _) in rec.groups)
    objs = [o for (_, o) in rec.groups]
    if every:   # a forced update carries the object after that group's solver step
        for a, b in zip(objs, objs[1:]):
            assert not numpy.array_equal(a, b)
        assert numpy.array_equal(objs[n_groups - 1], rec.iters[0][2])
        assert numpy.array_equal(objs[-1], state.object.data)
    else:   # otherwise the state as of the last iteration boundary
        assert all(numpy.array_equal(o, rec.start[0]) for o in objs[:n_groups])
        assert all(numpy.array_equal(o, rec.iters[0][2]) for o in objs[n_groups:])
    assert numpy.array_equal(rec.iters[-1][2], state.object.data)


class Stop(Exception):
    """Stands for the reference's EarlyTermination(state, continue_next_engine)."""

    def __init__(self, state):
        super().__init__('stop')
        self.state = state


class StopAt:
    """Ends the run at iteration k, as PatienceObserver does (observer.py:162-180)."""

    def __init__(self, k):
        self.k = k

    def update_iteration(self, state, i, n, error=None):
        if i == self.k:
            raise Stop(state)


def test_early_termination_hands_on_the_state_of_that_iteration():
    """execute_engine takes the state out of the exception (execute.py:83-89): it must be
    the state after the iteration that ended the run, not the one the engine started from."""
    c = make_case(seed=63, N=64, M=2, S=2, scan_shape=(5, 5))
    props = PL.ConventionalEnginePlan(
        noise_model={'type': 'amplitude', 'eps': 1e-2},
        solver={'type': 'lsqml', 'beta_object': 0.9, 'beta_probe': 0.8, 'gamma': 1e-3},
        niter=5, grouping=10, calc_error_fraction=1.0)
    with pytest.raises(Stop) as stop:
        run_conventional(run_args(c, StopAt(2), 'observer-seed'), props)
    state = stop.value.state
    assert state.iter.engine_iter == 2
    assert len(state.progress.detector_errors) == 2
    assert not numpy.array_equal(state.object.data, c.obj)
    assert not numpy.array_equal(state.probe.data, c.probe)
    assert numpy.isfinite(state.object.data).all()
