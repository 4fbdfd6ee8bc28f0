"""Batched amplitudes (QtreeSimulator.simulate_batch, qtensor/Simulate.py:66-94)
on the CPU: the reference fixtures against a dense state vector, the gate
conversion, and the compiled batch plans run by the CPU interpreter."""
import json
import os

import numpy as np
import pytest

import plan_interp
import statevector as sv
from conftest import ROOT
from qtensor_b200 import _lib
from qtensor_b200.plan import NetworkPlan
from qtensor_b200.simulator import gates_from_circuit

with open(os.path.join(ROOT, 'tests', 'golden', 'batch_reference.json')) as _f:
    CASES = json.load(_f)['cases']


class Gate:
    """Stand-in for a qtree gate object: name, qubits, parameters."""

    def __init__(self, name, qubits, alpha=None):
        self.name = name
        self.qubits = tuple(qubits)
        self.parameters = {} if alpha is None else {'alpha': alpha}


def circuit(case):
    return [Gate(n, q, a) for n, q, a in case['gates']]


def amplitudes(case, k):
    return np.array([complex(*z) for z in case['amplitudes'][str(k)]])


@pytest.mark.parametrize('ci', range(len(CASES)))
def test_fixture_matches_dense_state(ci):
    """The reference's batch order: qubit 0 is the most significant bit of
    the batch index, the other qubits are 0."""
    case = CASES[ci]
    n = case['n_qubits']
    psi = sv.circuit_state(case['gates'], n)
    for k in case['amplitudes']:
        k = int(k)
        want = psi[np.arange(2 ** k) << (n - k)]
        assert np.max(np.abs(amplitudes(case, k) - want)) < 1e-10


def test_gate_conversion():
    n, gates, params = gates_from_circuit([Gate('H', [0]), Gate('XPhase+', [1], 0.3), Gate('T+', [2]),
                                           Gate('ZZ', [0, 2], -0.7), Gate('cX', [2, 1]), Gate('I', [3])])
    assert n == 4
    assert list(gates['kind']) == [_lib.GATE_H, _lib.GATE_XPHASE, _lib.GATE_ZPHASE, _lib.GATE_ZZ, _lib.GATE_CX]
    assert list(gates['q0']) == [0, 1, 2, 0, 2] and list(gates['q1']) == [-1, -1, -1, 2, 1]
    assert np.allclose(params, [-0.3, -0.25, -0.7])
    with pytest.raises(NotImplementedError):
        gates_from_circuit([Gate('SWAP', [0, 1])])


@pytest.mark.parametrize('ci', range(len(CASES)))
def test_interpreted_batch_plans_match_reference(ci):
    case = CASES[ci]
    n, gates, params = gates_from_circuit(circuit(case))
    for k in case['amplitudes']:
        k = int(k)
        plan = NetworkPlan(len(params))
        first, group0 = plan.add_circuit_batch(max(n, k), gates, params, k)
        assert first == 0 and group0 == 0
        vals = plan_interp.run_plan(plan, params)
        assert len(vals) == 2 ** k
        assert np.max(np.abs(vals - amplitudes(case, k))) < 1e-12


def test_sliced_batch_plans_match_reference():
    """Batch outputs and slices together: every amplitude's slices sum to it."""
    case = CASES[2]
    n, gates, params = gates_from_circuit(circuit(case))
    probe = NetworkPlan(len(params))
    probe.add_circuit_batch(n, gates, params, 2)
    width = max(i['treewidth'] for i in probe.infos())
    plan = NetworkPlan(len(params))
    plan.set_max_width(width - 1)
    plan.add_circuit_batch(n, gates, params, 2)
    assert max(i['n_slices'] for i in plan.infos()) > 1
    assert max(i['treewidth'] for i in plan.infos()) < width
    vals = plan_interp.run_plan(plan, params)
    assert np.max(np.abs(vals - amplitudes(case, 2))) < 1e-12


def test_batch_vars_out_of_range():
    _, gates, params = gates_from_circuit(circuit(CASES[0]))
    plan = NetworkPlan(len(params))
    with pytest.raises(_lib.QtbError):
        plan.add_circuit_batch(4, gates, params, 5)
    with pytest.raises(_lib.QtbError):
        plan.add_circuit_batch(4, gates, params, -1)
