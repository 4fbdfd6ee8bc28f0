"""Property tests of the plan compiler on the CPU (derandomized hypothesis):
random graphs, depths and composers against the reference port edge by
edge, and random circuits (every supported gate and its dagger, slicing
forced or not, any batch of output qubits) against a dense state vector.
Plans run in the CPU interpreter with the device's encodings."""
import networkx as nx
import numpy as np
import pytest
from hypothesis import given, settings, strategies as st

import plan_interp
import qtensor_port as port
import statevector as sv
from qtensor_b200.lightcone import composer_id
from qtensor_b200.plan import NetworkPlan, graph_csr
from qtensor_b200.simulator import gates_from_circuit
from test_batch_amplitudes import Gate

SETTINGS = settings(max_examples=50, deadline=None, derandomize=True)


@st.composite
def qaoa_cases(draw):
    n = draw(st.integers(4, 12))
    seed = draw(st.integers(0, 10 ** 6))
    kind = draw(st.sampled_from(['regular', 'er', 'tree']))
    if kind == 'regular':
        G = nx.random_regular_graph(3, n + (n % 2), seed=seed)
    elif kind == 'er':
        G = nx.erdos_renyi_graph(n, 0.4, seed=seed)
    else:
        G = nx.random_labeled_tree(n, seed=seed) if hasattr(nx, 'random_labeled_tree') \
            else nx.random_tree(n, seed=seed)
    p = draw(st.integers(1, 2))
    rng = np.random.default_rng(seed)
    gamma = list(rng.uniform(0, np.pi, p))
    beta = list(rng.uniform(0, np.pi, p))
    comp = draw(st.sampled_from(['default', 'zz', 'cx']))
    return G, p, gamma, beta, comp


@SETTINGS
@given(qaoa_cases())
def test_random_graphs_match_reference(case):
    G, p, gamma, beta, comp = case
    if G.number_of_edges() == 0:
        return
    edges = list(G.edges())[:6]
    params = np.concatenate([gamma, beta])
    plan = NetworkPlan(2 * p)
    plan.set_order_trials(2)
    plan.add_lightcones(graph_csr(G), np.array(edges), p, composer_id(comp), params)
    vals = plan_interp.run_plan(plan, params)
    ref = np.array([complex(np.ravel(port.edge_energy(G, gamma, beta, e, composer=comp))[0])
                    for e in edges])
    assert np.max(np.abs(vals - ref)) < 1e-10


ONE = ['H', 'X', 'Y', 'Z', 'T', 'H+', 'T+']
ROT = ['ZPhase', 'XPhase', 'YPhase', 'ZPhase+', 'XPhase+', 'YPhase+']
TWO = ['cX', 'cZ', 'ZZ', 'ZZ+']


@st.composite
def circuits(draw):
    n = draw(st.integers(2, 6))
    gates = []
    for _ in range(draw(st.integers(4, 30))):
        kind = draw(st.sampled_from(['one', 'rot', 'two']))
        if kind == 'one':
            gates.append((draw(st.sampled_from(ONE)), [draw(st.integers(0, n - 1))], None))
        elif kind == 'rot':
            gates.append((draw(st.sampled_from(ROT)), [draw(st.integers(0, n - 1))],
                          draw(st.floats(-1, 1, allow_nan=False))))
        else:
            a, b = draw(st.lists(st.integers(0, n - 1), min_size=2, max_size=2, unique=True))
            name = draw(st.sampled_from(TWO))
            gates.append((name, [a, b], draw(st.floats(-1, 1, allow_nan=False)) if 'ZZ' in name else None))
    k = draw(st.integers(0, n))
    slice_to = draw(st.sampled_from([0, 2, 3]))
    return n, gates, k, slice_to


@SETTINGS
@given(circuits())
def test_random_circuits_match_dense_state(case):
    n, gates, k, slice_to = case
    qc = [Gate(name.rstrip('+') + ('+' if name.endswith('+') else ''), q, a) for name, q, a in gates]
    nq, garr, params = gates_from_circuit(qc)
    plan = NetworkPlan(len(params))
    if slice_to:
        plan.set_max_width(slice_to, 1 << 12)
    try:
        plan.add_circuit_batch(n, garr, params, k)
    except Exception as exc:      # a width the slice budget cannot reach
        assert slice_to and 'slice' in str(exc)
        return
    vals = plan_interp.run_plan(plan, params)
    psi = sv.circuit_state([(name, q, 0.0 if a is None else a) for name, q, a in gates], n)
    want = psi[np.arange(2 ** k) << (n - k)]
    assert np.max(np.abs(vals - want)) < 1e-10


@SETTINGS
@given(qaoa_cases())
def test_random_graphs_sliced_match_reference(case):
    """Slicing forced one below each circuit's width: the slices of an edge
    sum to the reference's term."""
    G, p, gamma, beta, comp = case
    if G.number_of_edges() == 0:
        return
    edges = list(G.edges())[:3]
    params = np.concatenate([gamma, beta])
    probe = NetworkPlan(2 * p)
    probe.add_lightcones(graph_csr(G), np.array(edges), p, composer_id(comp), params)
    width = max(i['treewidth'] for i in probe.infos())
    if width < 3:
        return
    plan = NetworkPlan(2 * p)
    plan.set_max_width(width, 1 << 12)
    plan.add_lightcones(graph_csr(G), np.array(edges), p, composer_id(comp), params)
    assert max(i['n_slices'] for i in plan.infos()) > 1
    vals = plan_interp.run_plan(plan, params)
    ref = np.array([complex(np.ravel(port.edge_energy(G, gamma, beta, e, composer=comp))[0])
                    for e in edges])
    assert np.max(np.abs(vals - ref)) < 1e-10
