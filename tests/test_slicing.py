"""Slicing choices of the plan compiler, checked on the CPU.

* Late slicing reproduces the reference's own ``LateParOptimizer``
  (qtensor/optimisation/late_parallelisation.py:30-202) exactly: its
  elimination order and its sliced variables, on the lightcones recorded in
  ``tests/golden/late_slicing_reference.json``.
* Tree trimming (``TreeTrimSplitter``, qtensor/optimisation/Optimizer.py:
  178-224; its qtree splitter is restated) brings the width to the target.
* Whatever the choice, the slices of a circuit sum to its amplitude: the
  compiled plans run in the numpy plan interpreter (complex128) match the
  reference's unsliced edge terms, as the reference's own
  ``test_qaoa_energy_feynman`` checks Feynman against plain energies
  (qtensor/tests/test_qaoa_energy.py:109-121).
"""
import json
import os

import numpy as np
import pytest

import graphs
import plan_interp
import qtensor_port as port
from conftest import ROOT, golden_graph
from qtensor_b200.lightcone import reference_lightcone, simplify_passes
from qtensor_b200.plan import NetworkPlan

LATE = os.path.join(ROOT, 'tests', 'golden', 'late_slicing_reference.json')


def _late_cases():
    with open(LATE) as f:
        return json.load(f)['cases']


def _compile(G, edge, p, params, method, max_width, trials=0, comp='default'):
    nq, gates = reference_lightcone(G, edge, p, comp)
    plan = NetworkPlan(2 * p)
    plan.set_order_trials(trials)
    plan.set_slicing(method)
    plan.set_max_width(max_width, 1024)
    plan.add_circuit(nq, gates, params, simplify_passes(comp))
    return plan, nq


@pytest.mark.parametrize('case', range(len(_late_cases())))
def test_late_slicing_matches_reference_late_par_optimizer(case):
    c = _late_cases()[case]
    G = graphs.regular(c['nodes'], seed=c['graph_seed'])
    gamma, beta = graphs.angles(c['p'], c['angle_seed'])
    plan, nq = _compile(G, tuple(c['edge']), c['p'], np.concatenate([gamma, beta]), 'late',
                        c['target_tw'] + 1)
    peo, k = plan.peo(0), len(c['sliced'])
    assert peo[2 * nq:len(peo) - k] == c['order']
    assert peo[len(peo) - k:] == c['sliced']
    assert plan.info(0)['n_slices'] == 2 ** k


@pytest.mark.parametrize('method', ['late', 'tree_trim', 'greedy'])
def test_sliced_plans_sum_to_the_reference_terms(method):
    """Every slicing choice, forced well below the width, on the N=20 p=1
    workload and the reference test families: the interpreted slices sum to
    the reference's edge terms."""
    for name, drop in (('cfg1_default', 2), ('test_random_n10_p5_d2', 3), ('test_grid2d_n3_p3_d0', 3)):
        G, w = golden_graph(name)
        p = len(w['gamma'])
        params = np.concatenate([w['gamma'], w['beta']])
        ref = np.array([complex(*t) for t in w['terms']])
        for k, edge in enumerate(G.edges()):
            width = w['widths'][k]
            if width - drop < 2:
                continue
            plan, _ = _compile(G, edge, p, params, method, width - drop + 1, comp=w['composer'])
            info = plan.info(0)
            assert info['n_slices'] > 1
            assert info['treewidth'] <= width - drop or method == 'late'
            vals = plan_interp.run_plan(plan, params)
            assert abs(vals[0] - ref[k]) < 1e-12


def test_tree_trimming_reaches_the_target_width():
    """TreeTrimSplitter's loop (Optimizer.py:183-224) ends at a width at
    most the target, on the N=10 p=3 problem of the reference's
    test_qaoa_energy_feynman with max_tw=13 (and tighter targets)."""
    G = graphs.regular(10, seed=1)
    gamma, beta = [np.pi / 3] * 3, [np.pi / 2] * 3
    params = np.concatenate([gamma, beta])
    for edge in list(G.edges())[:5]:
        for target in (13, 9, 7):
            plan, _ = _compile(G, edge, 3, params, 'tree_trim', target + 1, comp='cx')
            info = [plan.info(i) for i in range(len(plan))]
            assert max(i['treewidth'] for i in info) <= target
            amp = plan_interp.run_plan(plan, params)[0]
            circ = port.lightcone_circuit(G, edge, gamma, beta, 'cx')
            assert abs(amp - port.simulate_amplitude(circ)[0]) < 1e-12


def test_unknown_slicing_method_is_rejected():
    from qtensor_b200 import _lib
    plan = NetworkPlan(2)
    with pytest.raises(_lib.QtbError):
        _lib.check(plan._lib.qtb_plan_set_slicing(plan._h, 7))
