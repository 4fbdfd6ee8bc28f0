"""Generate the golden QAOA fixtures from the reference QTensor code.

Runs the reference package's own ``QAOAQtreeSimulator`` (imported from a
read-only reference checkout through ``oracle/refimport.py``, on the oracle
``qtree``) and writes ``qaoa_reference.json`` next to this script.  The GPU
box has no reference checkout; the tests read only the JSON.

    python tests/golden/make_golden.py [--skip-large]

Workloads (seeded; angles U[0, pi) from ``numpy.random.default_rng(seed)``):
  cfg1   3-regular N=20  p=1 seed 0 -- all three composers, per-edge terms,
         greedy widths and elimination orders
  cfg2   3-regular N=100 p=3 seed 0 -- per-edge terms (default composer)
  cfg3   3-regular N=1000 p=3 seed 0 -- per-edge terms (default composer)
  cfg4   3-regular N=256 p=4 seed 0 -- per-edge terms (default composer)
  tests  the graph families of qtensor/tests/test_qaoa_energy.py:36-43 with
         its angles gamma=pi/5, beta=pi/2 (seeded graphs)
  petersen  qtensor/tests/qiskit_qaoa_energy.py:112-123 angles, p=9
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
sys.path.insert(0, os.path.join(ROOT, 'tests'))

import graphs  # noqa: E402
from graphs import angles  # noqa: E402
from refimport import import_reference  # noqa: E402


def cplx(z):
    z = complex(np.asarray(z).reshape(-1)[0])
    return [z.real, z.imag]


def petersen():
    G = graphs.petersen()
    qiskit_params = np.array([
        5.192253984583296, 5.144373231492732, 5.9438949617723775, 5.807748946652058,
        3.533458907810596, 6.006206583282401, 6.122313961527631, 6.218468942101044,
        6.227704753217614, 0.3895570099244132, -0.1809282325810937, 0.8844522327007089,
        0.7916086532373585, 0.21294534589417236, 0.4328896243354414, 0.8327451563500539,
        0.7694639329585451, 0.4727893829336214])
    # qiskit rzz(theta) = ZZ(alpha=theta/pi), rx(theta) = XPhase(alpha=theta/pi)
    # (qtensor/tests/test_qaoa_energy.py:58, qiskit_qaoa_energy.py:107)
    gamma = list(qiskit_params[9:] / (2 * np.pi))
    beta = list(qiskit_params[:9] / np.pi)
    return G, gamma, beta


def main():
    qtensor = import_reference()
    if qtensor is None:
        sys.exit('no reference checkout found (set QTENSOR_REFERENCE)')
    from qtensor import (QAOAQtreeSimulator, DefaultQAOAComposer, QtreeQAOAComposer,
                         ZZQtreeQAOAComposer)
    composers = {'default': DefaultQAOAComposer, 'cx': QtreeQAOAComposer,
                 'zz': ZZQtreeQAOAComposer}

    def edge_terms(G, gamma, beta, comp='default', with_order=False):
        sim = QAOAQtreeSimulator(composers[comp])
        terms, widths, peos = [], [], []
        for edge in G.edges():
            terms.append(cplx(sim._get_edge_energy(G, gamma, beta, edge)))
            widths.append(int(sim.optimizer.treewidth))
            if with_order:
                peos.append([int(v) for v in sim.peo])
        return terms, widths, peos

    out = {'generator': 'tests/golden/make_golden.py', 'workloads': {}}
    skip_large = '--skip-large' in sys.argv

    def record(name, G, gamma, beta, comp='default', with_order=False, **extra):
        t0 = time.time()
        terms, widths, peos = edge_terms(G, gamma, beta, comp, with_order)
        total = sum(complex(*t) for t in terms)
        entry = {'n_nodes': G.number_of_nodes(), 'edges': [list(e) for e in G.edges()],
                 'gamma': gamma, 'beta': beta, 'composer': comp,
                 'terms': terms, 'widths': widths,
                 'energy': (G.number_of_edges() - total.real) / 2}
        if with_order:
            entry['peo'] = peos
        entry.update(extra)
        out['workloads'][name] = entry
        print('{:24s} energy {:.10f} max width {:2d} ({:.1f} s)'.format(
            name, entry['energy'], max(widths), time.time() - t0), flush=True)

    G = graphs.regular(20)
    g, b = angles(1, 0)
    for comp in composers:
        record('cfg1_' + comp, G, g, b, comp, with_order=True, graph='3-regular N=20 seed 0', p=1)

    fams = [(4, 4, 3, 'random'), (10, 5, 2, 'random'), (14, 1, 3, 'random'),
            (3, 3, 0, 'grid2d'), (8, 4, 0, 'line')]
    for n, p, d, kind in fams:
        Gt = graphs.family(kind, n, d)
        record('test_{}_n{}_p{}_d{}'.format(kind, n, p, d), Gt, [np.pi / 5] * p, [np.pi / 2] * p,
               graph='{} n={} d={} seed 1'.format(kind, n, d), p=p)

    Gp, gp, bp = petersen()
    record('petersen_p9', Gp, gp, bp, graph='Petersen', p=9, known_answer=12.0, tolerance=1e-2)

    G2 = graphs.regular(100)
    g, b = angles(3, 0)
    record('cfg2', G2, g, b, graph='3-regular N=100 seed 0', p=3)
    if not skip_large:
        G4 = graphs.regular(256)
        g, b = angles(4, 0)
        record('cfg4', G4, g, b, graph='3-regular N=256 seed 0', p=4)
        G3 = graphs.regular(1000)
        g, b = angles(3, 0)
        record('cfg3', G3, g, b, graph='3-regular N=1000 seed 0', p=3)

    with open(os.path.join(HERE, 'qaoa_reference.json'), 'w') as f:
        json.dump(out, f, separators=(',', ':'))


if __name__ == '__main__':
    main()
