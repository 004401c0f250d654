"""Host logic of the gradient engine (no GPU): solver splitting and variable
parsing as in phaser/engines/gradient/run.py:29-65 and phaser/types.py:280-302,
and the oracle's optax restatement against the published update rules."""
import numpy
import pytest

from oracle import phaser_np as P
from phaser_b200 import plan as PL
from phaser_b200.engines.gradient import process_solvers


def test_recons_vars_parses_comma_separated_strings():
    assert PL.recons_vars('object, probe') == frozenset({'object', 'probe'})
    assert PL.recons_vars(('positions',)) == frozenset({'positions'})
    with pytest.raises(ValueError):
        PL.recons_vars('object,wobble')


def test_process_solvers_splits_group_and_iteration_solvers():
    plan = PL.GradientEnginePlan(solvers={
        'object,probe': {'type': 'adam', 'learning_rate': 1e-2},
        'positions': {'type': 'sgd', 'learning_rate': 1.0, 'momentum': 0.9},
    })
    all_vars, group, per_iter = process_solvers(plan)
    assert all_vars == frozenset({'object', 'probe', 'positions'})
    assert [(vs, k) for (vs, k, _) in group] == [(frozenset({'object', 'probe'}), 'adam')]
    assert [(vs, k) for (vs, k, _) in per_iter] == [(frozenset({'positions'}), 'sgd')]
    assert group[0][2].b2 == 0.999 and per_iter[0][2].nesterov is True


def test_process_solvers_rejects_duplicates_and_mixed_sets():
    with pytest.raises(ValueError, match='Duplicate'):
        process_solvers(PL.GradientEnginePlan(solvers={
            'object': {'type': 'sgd', 'learning_rate': 1.0}, 'object,probe': {'type': 'sgd', 'learning_rate': 1.0}}))
    with pytest.raises(ValueError, match='per-iteration'):
        process_solvers(PL.GradientEnginePlan(solvers={'object,positions': {'type': 'sgd', 'learning_rate': 1.0}}))
    with pytest.raises(NotImplementedError):
        process_solvers(PL.GradientEnginePlan(solvers={'object': {'type': 'lbfgs'}}))
    with pytest.raises(TypeError):   # f_min has no default (phaser/plan.py:161-165)
        process_solvers(PL.GradientEnginePlan(solvers={'object': {'type': 'polyak_sgd', 'max_learning_rate': 1.}}))


def test_oracle_adam_first_step_is_normalised_direction():
    d = numpy.array([3 + 4j, -1e-3j, 0], numpy.complex128)
    opt = P.OptaxNP('adam', {'learning_rate': 0.1, 'eps': 1e-8}, {'o': d})
    u = opt.update({'o': d}, 0.0)['o']
    assert numpy.allclose(u, 0.1 * d / (numpy.abs(d) + 1e-8))


def test_oracle_sgd_nesterov_trace():
    d1, d2 = numpy.array([1.0, -2.0]), numpy.array([0.5, 0.25])
    opt = P.OptaxNP('sgd', {'learning_rate': 0.1, 'momentum': 0.9, 'nesterov': True}, {'p': d1})
    u1 = opt.update({'p': d1}, 0.0)['p']
    u2 = opt.update({'p': d2}, 0.0)['p']
    t2 = d2 + 0.9 * d1
    assert numpy.allclose(u1, 0.1 * (d1 + 0.9 * d1))
    assert numpy.allclose(u2, 0.1 * (d2 + 0.9 * t2))


def test_oracle_polyak_step_is_capped_and_zero_for_zero_gradient():
    d = numpy.array([1.0, 1.0])
    opt = P.OptaxNP('polyak_sgd', {'max_learning_rate': 0.25, 'f_min': 0.0, 'scaling': 1.0}, {'p': d})
    assert numpy.allclose(opt.update({'p': d}, 0.2)['p'], 0.1 * d)     # (0.2 - 0) / 2
    assert numpy.allclose(opt.update({'p': d}, 10.0)['p'], 0.25 * d)   # capped
    assert numpy.all(opt.update({'p': 0 * d}, 1.0)['p'] == 0)
