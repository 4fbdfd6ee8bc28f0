"""CPU port of QTensor's QAOA edge-energy path on the oracle ``qtree``.

TEST INFRASTRUCTURE ONLY (the checker and the timed CPU reference arm): the
``qtensor_b200`` product never imports this module.

Restates, on top of ``oracle/qtree``:

* ``qtensor/utils.py:176-189``           -- ``nodes_at_distance`` / ``get_edge_subgraph``;
* ``qtensor/CircuitComposer.py:82-96,131-169`` -- the lightcone ``U Z_i Z_j U^+``
  circuit of ``QAOAComposer`` / ``ZZQAOAComposer`` (cone ansatz with layer l
  acting on the radius ``p-l`` subgraph, ``energy_edge``, inverse);
* ``qtensor/OpFactory.py:44-58,157-158`` -- the compact diagonal ``ZZ`` gate and
  ``QtreeBuilder.inverse`` (reversed daggers);
* ``qtensor/simplify_circuit/simplify_circuit.py:30-138`` and
  ``simplify_circuit_api.py:74-106`` -- commutation-based merge/cancel, used by
  ``DefaultQAOAComposer`` (``qtensor/__init__.py:55-63``);
* ``qtensor/optimisation/TensorNet.py:47-68``, ``qtensor/utils.py:12-44,77-87``,
  ``qtensor/optimisation/Optimizer.py:50-87`` -- tensor net, line graph and
  greedy min-degree ordering;
* ``qtensor/Simulate.py:36-100`` -- ``QtreeSimulator.simulate_batch``;
* ``qtensor/QAOASimulator.py:16-88`` -- per-edge energies, the process-pool
  variant and MaxCut post-processing;
* ``qtensor/ProcessingFrameworks.py:23-37`` -- ``NumpyBackend``.
"""
import itertools
import os
from multiprocessing import get_context

import networkx as nx
import numpy as np

from qtree import operators as qops
from qtree import optimizer as qopt
from qtree import np_framework, utils as qutils, graph_model


# --------------------------------------------------------------------------
# gates
# --------------------------------------------------------------------------
class ZZ(qops.ParametricGate):
    """Diagonal ``exp(-i pi alpha/2 Z Z)`` on two existing variables
    (``qtensor/OpFactory.py:44-58``)."""
    name = 'ZZ'
    _changes_qubits = ()
    parameter_count = 1

    def gen_tensor(self):
        a = self._parameters['alpha']
        m, p = np.exp(-1j * np.pi * a / 2), np.exp(1j * np.pi * a / 2)
        return np.array([[m, p], [p, m]])


# --------------------------------------------------------------------------
# lightcone
# --------------------------------------------------------------------------
def nodes_at_distance(G, nodes, dist):
    """Nodes within ``dist`` hops (``qtensor/utils.py:176-185``); the set
    bookkeeping is kept as in the reference because its iteration order
    fixes the qubit numbering of the cone."""
    nodes = list(nodes)
    for _ in range(dist):
        grown = list(nodes)
        for n in nodes:
            grown += list(G[n].keys())
        nodes = list(set(grown))
    return set(nodes)


def get_edge_subgraph(G, edge, dist):
    return G.subgraph(set(nodes_at_distance(G, edge, dist)))


def _cone_ansatz(cone, edge, gamma, beta, zz):
    """Hadamards, then for layer ``l`` (radius ``p-l``) the cost and mixer
    terms (``qtensor/CircuitComposer.py:138-151``)."""
    gates = [qops.H(q) for q in range(cone.number_of_nodes())]
    p = len(gamma)
    for radius, g, b in zip(range(p, 0, -1), gamma, beta):
        layer = get_edge_subgraph(cone, edge, radius)
        for u, v in layer.edges():
            if zz:
                gates.append(ZZ(u, v, alpha=2 * g))
            else:
                gates += [qops.cX(u, v), qops.ZPhase(v, alpha=2 * g), qops.cX(u, v)]
        for n in layer.nodes():
            gates.append(qops.XPhase(n, alpha=2 * b))
    return gates


def lightcone_circuit(G, edge, gamma, beta, composer='default'):
    """Gate list of ``<psi| Z_i Z_j |psi>`` restricted to the edge's lightcone.

    ``composer``: ``'default'`` (ZZ gates + simplification, applied twice as the
    reference's ``SimpZZQtreeComposer.circuit`` property is read twice on this
    path: ``CircuitComposer.py:95`` and ``QAOASimulator.py:24``), ``'zz'``
    (``ZZQtreeQAOAComposer``) or ``'cx'`` (``QtreeQAOAComposer``).
    """
    if len(gamma) != len(beta):
        raise ValueError('gamma and beta must have the same length')
    sub = get_edge_subgraph(G, edge, len(gamma))
    mapping = {v: k for k, v in enumerate(sub.nodes())}
    cone = nx.relabel_nodes(sub, mapping, copy=True)
    e = (mapping[edge[0]], mapping[edge[1]])
    zz = composer in ('default', 'zz')
    first = _cone_ansatz(cone, e, gamma, beta, zz) + [qops.Z(e[0]), qops.Z(e[1])]
    second = [g.dagger_me() for g in _cone_ansatz(cone, e, gamma, beta, zz)][::-1]
    circuit = first + second
    if composer == 'default':
        circuit = simplify_qtree_circuit(simplify_qtree_circuit(circuit))
    return circuit


# --------------------------------------------------------------------------
# simplifier (qtensor/simplify_circuit/)
# --------------------------------------------------------------------------
class _SGate:
    """Commutation record: kind, acted-on qubits, per-qubit eigenbasis, angle
    (``qtensor/simplify_circuit/gates.py``)."""
    __slots__ = ('kind', 'index', 'basis', 'angle')

    def __init__(self, kind, index, angle):
        self.kind = kind
        if kind == 'zz':
            self.index = tuple(sorted(index))
            self.basis = {q: 'Z' for q in index}
            self.angle = angle
        elif kind in ('x', 'y', 'zp'):
            self.index = tuple(index)
            self.basis = {index[0]: {'x': 'X', 'y': 'Y', 'zp': 'Z'}[kind]}
            self.angle = angle
        elif kind == 'z':
            self.index = tuple(index)
            self.basis = {index[0]: 'Z'}
            self.angle = 0
        elif kind == 'h':
            self.index = tuple(index)
            self.basis = {index[0]: 'X+Y'}
            self.angle = np.pi / 2 / np.sqrt(2)  # constant, whatever is passed
        elif kind == 'cx':
            self.index = tuple(index)
            self.basis = {index[0]: 'cnot_A', index[1]: 'cnot_B'}
            self.angle = 0
        elif kind == 'id':
            self.index = ()
            self.basis = {}
            self.angle = 0
        else:
            raise ValueError(kind)


_KIND_OF = {ZZ: 'zz', qops.XPhase: 'x', qops.YPhase: 'y', qops.ZPhase: 'zp',
            qops.H: 'h', qops.cX: 'cx', qops.Z: 'z'}
_GATE_OF = {v: k for k, v in _KIND_OF.items()}


def _commute(a, b):
    return all(a.basis[q] == b.basis[q] for q in set(a.index) & set(b.index))


def simplify_circuit(gates):
    """Merge/cancel equal-kind gate pairs on the same qubits whose in-between
    gates commute with the first one; pairs are visited by increasing
    distance (``np.argsort`` of the distances, as the reference), a pair whose
    angles sum below 1e-5 cancels (``simplify_circuit.py:50-138``)."""
    if not gates:
        return []
    cir = list(gates)
    pairs = [(i, j) for i in range(len(cir) - 1) for j in range(i + 1, len(cir))
             if cir[i].kind == cir[j].kind and cir[i].index == cir[j].index]
    if not pairs:
        return cir
    order = np.argsort(np.diff(np.array(pairs), 1)[:, 0])
    for k in order:
        a, b = pairs[k]
        if cir[a].kind == 'id' or cir[b].kind == 'id':
            continue
        if all(_commute(cir[a], cir[m]) for m in range(a + 1, b)):
            total = cir[a].angle + cir[b].angle
            if abs(total) < 1e-5:
                cir[a], cir[b] = _SGate('id', (), 0), _SGate('id', (), 0)
            else:
                cir[a], cir[b] = _SGate('id', (), 0), _SGate(cir[a].kind, cir[a].index, total)
    return [g for g in cir if g.kind != 'id']


def simplify_qtree_circuit(circuit):
    """qtree gates -> commutation records -> simplified qtree gates
    (``simplify_circuit_api.py:74-106``); daggered parametric gates enter with
    the sign of ``alpha`` flipped and leave as plain gates."""
    records = []
    for g in circuit:
        kind = _KIND_OF[type(g)]
        if 'alpha' in g.parameters:
            sign = -1 if '+' in g.name else 1
            records.append(_SGate(kind, g.qubits, sign * g.parameters['alpha']))
        else:
            records.append(_SGate(kind, g.qubits, 0))
    out = []
    for r in simplify_circuit(records):
        cls = _GATE_OF[r.kind]
        if issubclass(cls, qops.ParametricGate):
            out.append(cls(*r.index, alpha=r.angle))
        else:
            out.append(cls(*r.index))
    return out


# --------------------------------------------------------------------------
# tensor network, ordering, simulation
# --------------------------------------------------------------------------
class NumpyBackend:
    """``qtensor/ProcessingFrameworks.py:23-37``."""

    def process_bucket(self, bucket, no_sum=False):
        return np_framework.process_bucket_np(bucket, no_sum=no_sum)

    def get_sliced_buckets(self, buckets, data_dict, slice_dict):
        return np_framework.get_sliced_np_buckets(buckets, data_dict, slice_dict)

    def get_result_data(self, result):
        return result.data


def circuit_to_network(circuit):
    """``QtreeTensorNet.from_qtree_gates`` (``TensorNet.py:60-68``)."""
    n_qubits = len(set(q for g in circuit for q in g.qubits))
    return qopt.circ2buckets(n_qubits, [[g] for g in circuit])


def greedy_order(graph):
    """Min-degree elimination order (``qtensor/utils.py:12-44``): repeatedly
    take the first node (graph node order) with the fewest distinct
    neighbours, connect its neighbours, remove it.  Returns (peo, degrees)."""
    nodes = list(graph.nodes())
    adj = {n: set(graph[n]) - {n} for n in nodes}
    alive = list(nodes)
    peo, degrees = [], []
    while alive:
        best = min(range(len(alive)), key=lambda k: (len(adj[alive[k]]), k))
        node = alive.pop(best)
        nbrs = adj.pop(node)
        peo.append(node)
        degrees.append(len(nbrs))
        for a in nbrs:
            adj[a].discard(node)
        for a, b in itertools.combinations(nbrs, 2):
            adj[a].add(b)
            adj[b].add(a)
    return peo, degrees


def order_network(buckets, bra_vars, ket_vars):
    """``OrderingOptimizer.optimize`` without free variables
    (``Optimizer.py:65-87``): peo = ket + bra + greedy order of the rest."""
    ignored = ket_vars + bra_vars
    graph = graph_model.buckets2graph(buckets, ignore_variables=ignored)
    peo_ints, degrees = greedy_order(graph)
    peo = [qopt.Var(v, size=graph.nodes[v]['size'], name=graph.nodes[v]['name'])
           for v in peo_ints]
    return ignored + peo, (max(degrees) if degrees else 0)


def simulate_amplitude(circuit, backend=None, return_width=False):
    """``QtreeSimulator.simulate`` (``Simulate.py:66-100``) with
    ``batch_vars=0``: the amplitude ``<0|circuit|0>``."""
    backend = backend or NumpyBackend()
    buckets, data_dict, bra, ket = circuit_to_network(circuit)
    peo, width = order_network(buckets, bra, ket)
    buckets, perm = qopt.reorder_buckets(buckets, peo)
    ket = sorted([perm[v] for v in ket], key=str)
    bra = sorted([perm[v] for v in bra], key=str)
    slice_dict = qutils.slice_from_bits(0, ket)
    slice_dict.update(qutils.slice_from_bits(0, bra))
    sliced = backend.get_sliced_buckets(buckets, data_dict, slice_dict)
    result = qopt.bucket_elimination(sliced, backend.process_bucket, n_var_nosum=0)
    amp = np.asarray(backend.get_result_data(result)).flatten()
    return (amp, width) if return_width else amp


def edge_energy(G, gamma, beta, edge, composer='default', backend=None):
    """``QAOASimulator._get_edge_energy`` (``QAOASimulator.py:16-24``)."""
    return simulate_amplitude(lightcone_circuit(G, edge, gamma, beta, composer), backend)


def post_process_energy(G, E):
    """``QAOASimulator._post_process_energy`` (``QAOASimulator.py:27-41``):
    MaxCut cost ``(|E| - Re sum <Z_i Z_j>) / 2``."""
    return (G.number_of_edges() - np.real(E)) / 2


def energy_expectation(G, gamma, beta, composer='default', backend=None):
    """Serial sum over edges (``QAOASimulator.py:44-66``)."""
    total = 0
    for edge in G.edges():
        total = total + edge_energy(G, gamma, beta, edge, composer, backend)
    return post_process_energy(G, total)


def _edge_task(args):
    G, gamma, beta, edge, composer = args
    return edge_energy(G, gamma, beta, edge, composer)


def energy_expectation_parallel(G, gamma, beta, n_processes=None, composer='default',
                                edges=None, start_method='spawn'):
    """Process-pool variant (``QAOASimulator.py:72-88``).  The default
    ``spawn`` pool is safe in a process that already initialised CUDA; pass
    ``'fork'`` only before any GPU call.  ``edges`` limits the work to a
    subset (returns the raw sum of edge terms in that case)."""
    n_processes = n_processes or os.cpu_count()
    todo = list(G.edges()) if edges is None else list(edges)
    args = [(G, gamma, beta, e, composer) for e in todo]
    with get_context(start_method).Pool(n_processes) as pool:
        terms = pool.map(_edge_task, args, chunksize=max(1, len(args) // (4 * n_processes)))
    total = sum(terms)
    if edges is not None:
        return total
    return post_process_energy(G, total)
