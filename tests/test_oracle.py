"""The oracle pinned against the reference's golden fixtures and independent
physics (CPU only)."""
import networkx as nx
import numpy as np
import pytest

import graphs
import qtensor_port as port
import statevector as sv
from conftest import golden, golden_graph
from refimport import import_reference


def _terms(w):
    return np.array([complex(*t) for t in w['terms']])


@pytest.mark.parametrize('comp', ['default', 'cx', 'zz'])
def test_port_matches_reference_cfg1(comp):
    """Per-edge amplitudes, widths and elimination orders of the reference
    (run on the oracle qtree) are reproduced by the port."""
    G, w = golden_graph('cfg1_' + comp)
    gamma, beta = w['gamma'], w['beta']
    ref = _terms(w)
    for k, edge in enumerate(G.edges()):
        circ = port.lightcone_circuit(G, edge, gamma, beta, comp)
        amp, width = port.simulate_amplitude(circ, return_width=True)
        assert abs(amp[0] - ref[k]) < 1e-12
        assert width == w['widths'][k]
        buckets, _, bra, ket = port.circuit_to_network(circ)
        peo, _ = port.order_network(buckets, bra, ket)
        assert [int(v) for v in peo] == w['peo'][k]
    E = port.energy_expectation(G, gamma, beta, comp)
    assert abs(E[0] - w['energy']) < 1e-10


@pytest.mark.parametrize('name', ['test_random_n4_p4_d3', 'test_random_n10_p5_d2',
                                  'test_random_n14_p1_d3', 'test_grid2d_n3_p3_d0',
                                  'test_line_n8_p4_d0'])
def test_port_matches_reference_families(name):
    G, w = golden_graph(name)
    E = port.energy_expectation(G, w['gamma'], w['beta'])
    assert abs(E[0] - w['energy']) < 1e-10


def test_petersen_known_answer():
    """qtensor/tests/qiskit_qaoa_energy.py:112-123: |E| = 12 within 1e-2."""
    G, w = golden_graph('petersen_p9')
    assert abs(w['energy'] - 12.0) < 1e-2
    assert abs(sv.qaoa_energy_statevector(G, w['gamma'], w['beta']) - w['energy']) < 1e-10


@pytest.mark.parametrize('name', ['cfg1_default', 'test_random_n4_p4_d3', 'test_random_n10_p5_d2',
                                  'test_random_n14_p1_d3', 'test_grid2d_n3_p3_d0',
                                  'test_line_n8_p4_d0'])
def test_golden_matches_statevector(name):
    """The reference's energies agree with a dense state vector."""
    G, w = golden_graph(name)
    assert abs(sv.qaoa_energy_statevector(G, w['gamma'], w['beta']) - w['energy']) < 1e-9


def test_golden_matches_p1_closed_form():
    G, w = golden_graph('cfg1_default')
    for k, edge in enumerate(G.edges()):
        exact = sv.qaoa_p1_edge_term(G, edge, w['gamma'][0], w['beta'][0])
        assert abs(complex(*w['terms'][k]) - exact) < 1e-12


@pytest.mark.parametrize('name,stride', [('cfg2', 15), ('cfg3', 150), ('cfg4', 64)])
def test_port_matches_reference_large(name, stride):
    """A sample of the large workloads' edges, port vs reference fixture."""
    G, w = golden_graph(name)
    edges = list(G.edges())
    for k in range(0, len(edges), stride):
        amp = port.edge_energy(G, w['gamma'], w['beta'], edges[k])
        assert abs(amp[0] - complex(*w['terms'][k])) < 1e-12


def test_planted_mistake_is_caught():
    """A wrong ZZ sign in the oracle moves the energy far beyond tolerance."""
    G, w = golden_graph('cfg1_default')
    good = port.energy_expectation(G, w['gamma'], w['beta'])[0]
    orig = port.ZZ.gen_tensor

    def wrong(self):
        return orig(self).conj()
    port.ZZ.gen_tensor = wrong
    try:
        bad = port.energy_expectation(G, w['gamma'], w['beta'])[0]
    finally:
        port.ZZ.gen_tensor = orig
    assert abs(good - w['energy']) < 1e-10
    assert abs(bad - w['energy']) > 1e-3


def test_port_matches_live_reference():
    """Where a reference checkout exists, its simulator and the port agree."""
    qtensor = import_reference()
    if qtensor is None:
        pytest.skip('no reference checkout on this machine')
    G = graphs.regular(12, seed=3)
    gamma, beta = graphs.angles(2, seed=3)
    sim = qtensor.QAOAQtreeSimulator(qtensor.DefaultQAOAComposer)
    ref = sim.energy_expectation(G, gamma, beta)
    assert abs(ref[0] - port.energy_expectation(G, gamma, beta)[0]) < 1e-12


def test_golden_fixture_is_complete():
    names = set(golden())
    for want in ('cfg1_default', 'cfg1_cx', 'cfg1_zz', 'cfg2', 'cfg3', 'cfg4', 'petersen_p9'):
        assert want in names


def test_slice_digits_beyond_numpy_rank():
    """The oracle's slice_from_bits serves lightcones of more than 64 qubits
    (numpy's unravel_index stops at 64 dimensions) with the same digits."""
    from qtree.utils import unravel_index
    for v, dims in ((0, (2, 2, 2)), (5, (2, 2, 2)), (7, (2, 3, 2)), (23, (3, 4, 2))):
        assert unravel_index(v, dims) == tuple(int(x) for x in np.unravel_index(v, dims))
    assert unravel_index(0, (2,) * 89) == (0,) * 89
    assert unravel_index(2 ** 88 + 1, (2,) * 89) == (1,) + (0,) * 87 + (1,)


def test_wide_request_fixture_rebuilds():
    """The wide serving request of tests/golden/wide_request_reference.json
    is rebuilt from its seeds, and its recorded widths are the reference
    greedy widths of the port."""
    import json
    import os
    from conftest import ROOT
    with open(os.path.join(ROOT, 'tests', 'golden', 'wide_request_reference.json')) as f:
        w = json.load(f)
    G = graphs.erdos_renyi(w['graph']['n'], w['graph']['seed'])
    assert [list(e) for e in G.edges()] == w['edges']
    assert list(graphs.angles(3, w['graph']['angle_seed'])[0]) == w['gamma']
    for i in (0, 1, 2):
        circ = port.lightcone_circuit(G, tuple(w['edges'][i]), w['gamma'], w['beta'])
        buckets, _, bra, ket = port.circuit_to_network(circ)
        assert port.order_network(buckets, bra, ket)[1] == w['widths'][i]
