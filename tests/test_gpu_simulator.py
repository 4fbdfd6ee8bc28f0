"""QtreeSimulator on the GPU against the reference's simulate_batch fixtures
(seeded random circuits of H, X, Y, Z, T, cX, cZ, ZPhase, XPhase, YPhase,
ZZ and their daggers; batch_vars up to 5), with and without slicing."""
import numpy as np
import pytest

from test_batch_amplitudes import CASES, Gate, amplitudes, circuit

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.mark.parametrize('ci', range(len(CASES)))
def test_simulate_batch_matches_reference(cuda_device, ci):
    from qtensor_b200.simulator import QtreeSimulator
    case = CASES[ci]
    sim = QtreeSimulator()
    for k in case['amplitudes']:
        got = sim.simulate_batch(circuit(case), batch_vars=int(k))
        assert np.max(np.abs(got - amplitudes(case, int(k)))) < TOL
    state = sim.simulate(circuit(case))
    assert state.shape == (1,) and abs(state[0] - amplitudes(case, 0)[0]) < TOL


def test_simulate_batch_sliced(cuda_device):
    from qtensor_b200.simulator import QtreeSimulator
    case = CASES[2]
    got = QtreeSimulator(max_width=3).simulate_batch(circuit(case), batch_vars=2)
    assert np.max(np.abs(got - amplitudes(case, 2))) < TOL


def test_simulator_errors_like_reference(cuda_device):
    from qtensor_b200.simulator import QtreeSimulator
    case = CASES[1]
    with pytest.raises(ValueError, match='max_tw'):
        QtreeSimulator(max_tw=1).simulate_batch(circuit(case), batch_vars=1)
    with pytest.raises(NotImplementedError):
        QtreeSimulator().simulate_batch(circuit(case), peo=[0, 1])
    with pytest.raises(NotImplementedError):
        QtreeSimulator().simulate([Gate('SWAP', [0, 1])])


def test_feynman_simulator_matches_reference(cuda_device):
    """FeynmanSimulator semantics: sliced below max_tw - tw_bias, paths summed."""
    from qtensor_b200.simulator import FeynmanSimulator
    case = CASES[2]
    sim = FeynmanSimulator(max_tw=5, n_processes=4)
    got = sim.simulate(circuit(case), batch_vars=2, tw_bias=2)
    assert np.max(np.abs(got - amplitudes(case, 2))) < TOL
    got0 = FeynmanSimulator().simulate_batch_adaptive(circuit(case))
    assert abs(got0[0] - amplitudes(case, 0)[0]) < TOL


def test_idle_qubits_and_empty_circuits(cuda_device):
    """Qubits without gates contribute <b|0> (the measurement tensor joins
    their bra and ket variables), as in the reference's circ2buckets."""
    import statevector as sv
    from qtensor_b200 import _lib
    from qtensor_b200.simulator import QtreeSimulator
    sim = QtreeSimulator()
    gates = [('H', [2], None), ('cX', [2, 0], None)]
    got = sim.simulate_batch([Gate(*g) for g in gates], batch_vars=3)
    assert np.max(np.abs(got - sv.circuit_state(gates, 3))) < TOL
    empty = sim.simulate_batch(np.zeros(0, dtype=_lib.GATE_DTYPE), batch_vars=2)
    assert np.max(np.abs(empty - np.array([1, 0, 0, 0]))) < TOL
