"""Edge terms of a wide serving request from the oracle port (complex128).

The request is the Erdos-Renyi graph N=213 (mean degree 3, seed 796350419)
at p=3 of the serving workload's stream: its widest lightcones have a
reference greedy width of 31 and more, and the engine compiles them only by
slicing.  The port of the reference's path (``oracle/qtensor_port.py``: the
reference's circuits, bucket layout, greedy order and NumpyBackend einsum
in complex128) contracts every edge whose reference greedy width is at most
``PORT_MAX_WIDTH`` (2^26 complex128 = 1 GB tensors; the widest ones two at a
time to bound host memory); their terms go to ``wide_request_reference.json``,
with each edge's reference width.  Edges above that width (28 to 35) are
listed without terms: the port would need tensors of 2^28 to 2^35 elements.

    python tests/golden/make_wide_golden.py
"""
import json
import os
import sys
import time
from multiprocessing import get_context

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
sys.path.insert(0, os.path.join(ROOT, 'tests'))

import graphs  # noqa: E402
import qtensor_port as port  # noqa: E402

GRAPH = dict(n=213, seed=796350419, p=3, angle_seed=656419913)
PORT_MAX_WIDTH = 26
SMALL_WIDTH = 24


def request():
    G = graphs.erdos_renyi(GRAPH['n'], GRAPH['seed'])
    gamma, beta = graphs.angles(GRAPH['p'], GRAPH['angle_seed'])
    return G, gamma, beta


def edge_width(args):
    G, gamma, beta, edge = args
    circ = port.lightcone_circuit(G, edge, gamma, beta)
    buckets, _, bra, ket = port.circuit_to_network(circ)
    _, width = port.order_network(buckets, bra, ket)
    return width


def edge_term(args):
    G, gamma, beta, edge = args
    return complex(port.edge_energy(G, gamma, beta, edge)[0])


def main():
    G, gamma, beta = request()
    edges = list(G.edges())
    t0 = time.time()
    with get_context('spawn').Pool(os.cpu_count()) as pool:
        widths = pool.map(edge_width, [(G, gamma, beta, e) for e in edges])
        small = [i for i, w in enumerate(widths) if w <= SMALL_WIDTH]
        terms = pool.map(edge_term, [(G, gamma, beta, edges[i]) for i in small], chunksize=1)
    large = [i for i, w in enumerate(widths) if SMALL_WIDTH < w <= PORT_MAX_WIDTH]
    with get_context('spawn').Pool(2) as pool:
        terms += pool.map(edge_term, [(G, gamma, beta, edges[i]) for i in large], chunksize=1)
    todo = small + large
    out = {'generator': 'tests/golden/make_wide_golden.py', 'graph': GRAPH, 'gamma': gamma, 'beta': beta,
           'edges': [list(e) for e in edges], 'widths': widths, 'port_max_width': PORT_MAX_WIDTH,
           'terms': {str(i): [t.real, t.imag] for i, t in zip(todo, terms)}}
    with open(os.path.join(HERE, 'wide_request_reference.json'), 'w') as f:
        json.dump(out, f, separators=(',', ':'))
    print('{} edges, {} with port terms, widest {} ({:.0f} s)'.format(
        len(edges), len(todo), max(widths), time.time() - t0))


if __name__ == '__main__':
    main()
