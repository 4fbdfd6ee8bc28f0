"""QAOA lightcone circuits as plan-compiler gate arrays.

Two qubit orders are offered:

* ``'native'`` -- built by the C++ plan compiler (``qtb_plan_add_lightcones``):
  cone qubits in increasing node id, layer edges in increasing (a, b) order;
  multithreaded, no Python per edge.
* ``'reference'`` -- built here with the same networkx operations as the
  reference composer, so qubit numbering, gate order and therefore the
  greedy elimination order are identical to QTensor's:
  ``get_edge_subgraph`` (qtensor/utils.py:176-189), the relabelled cone
  (qtensor/CircuitComposer.py:82-96), the per-layer radius subgraphs of
  ``QAOAComposer.cone_ansatz`` (qtensor/CircuitComposer.py:138-151), Z on the
  edge, and the reversed daggered ansatz (qtensor/OpFactory.py:157-158).
"""
import networkx as nx
import numpy as np

from . import _lib

COMPOSERS = {'default': _lib.COMPOSER_DEFAULT, 'zz': _lib.COMPOSER_ZZ, 'cx': _lib.COMPOSER_CX}


def composer_id(composer):
    if isinstance(composer, int):
        return composer
    try:
        return COMPOSERS[composer]
    except KeyError:
        raise ValueError('unknown composer {!r}; expected one of {}'.format(
            composer, sorted(COMPOSERS))) from None


def _ball(G, edge, radius):
    """Nodes within ``radius`` hops of ``edge``.  Each round appends every
    member's neighbours and deduplicates through a ``set``; the resulting set
    iteration order is what numbers the reference's cone qubits."""
    members = list(edge)
    for _ in range(radius):
        members = list(set(members + [w for v in members for w in G[v]]))
    return set(members)


def _subgraph_around(G, edge, radius):
    return G.subgraph(set(_ball(G, edge, radius)))


def reference_lightcone(G, edge, p, composer='default'):
    """``(n_qubits, gates)`` of the edge's ``<psi|Z_u Z_v|psi>`` circuit in the
    reference's qubit order; params are ``gamma[0..p), beta[0..p)``."""
    cid = composer_id(composer)
    sub = _subgraph_around(G, edge, p)
    index = {v: k for k, v in enumerate(sub.nodes())}
    cone = nx.relabel_nodes(sub, index, copy=True)
    e = (index[edge[0]], index[edge[1]])
    ansatz = [(_lib.GATE_H, q, -1, -1, 0.0) for q in range(cone.number_of_nodes())]
    for layer, radius in enumerate(range(p, 0, -1)):
        shell = _subgraph_around(cone, e, radius)
        for a, b in shell.edges():
            if cid == _lib.COMPOSER_CX:
                ansatz += [(_lib.GATE_CX, a, b, -1, 0.0),
                           (_lib.GATE_ZPHASE, b, -1, layer, 2.0),
                           (_lib.GATE_CX, a, b, -1, 0.0)]
            else:
                ansatz.append((_lib.GATE_ZZ, a, b, layer, 2.0))
        ansatz += [(_lib.GATE_XPHASE, q, -1, p + layer, 2.0) for q in shell.nodes()]
    gates = list(ansatz)
    gates += [(_lib.GATE_Z, e[0], -1, -1, 0.0), (_lib.GATE_Z, e[1], -1, -1, 0.0)]
    gates += [(k, a, b, prm, -c) for (k, a, b, prm, c) in reversed(ansatz)]
    return cone.number_of_nodes(), np.array(gates, dtype=_lib.GATE_DTYPE)


def simplify_passes(composer):
    """The default composer's circuit is read through the simplifying
    ``SimpZZQtreeComposer.circuit`` property twice on the energy path
    (qtensor/CircuitComposer.py:95 and qtensor/QAOASimulator.py:24)."""
    return 2 if composer_id(composer) == _lib.COMPOSER_DEFAULT else 0
