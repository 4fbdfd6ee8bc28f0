"""Record the reference's LateParOptimizer choices on QAOA lightcones.

Runs the reference's ``LateParOptimizer`` (qtensor/optimisation/
late_parallelisation.py:30-202; imported from a read-only reference checkout
through ``oracle/refimport.py``, on the oracle ``qtree``) on the lightcone
tensor networks of seeded 3-regular graphs, with ``target_tw`` two and three
below the reference greedy width, and writes the elimination order (its
contracted prefixes, then the rest) and the sliced variables to
``late_slicing_reference.json``.  The reference's ``optimize`` prepends the
ket and bra variables to the first bunch's slice list (:197-199); they are
not sliced, so the fixture keeps only the other variables.

    python tests/golden/make_slicing_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
sys.path.insert(0, os.path.join(ROOT, 'tests'))

import graphs  # noqa: E402
from refimport import import_reference  # noqa: E402

CASES = [
    # graph nodes, graph seed, p, angle seed, edges
    (30, 2, 3, 2, 6),
    (24, 5, 3, 5, 4),
    (16, 7, 4, 7, 3),
]


def main():
    qtensor = import_reference()
    if qtensor is None:
        sys.exit('no reference checkout found (set QTENSOR_REFERENCE)')
    from qtensor import DefaultQAOAComposer
    from qtensor.optimisation.Optimizer import OrderingOptimizer
    from qtensor.optimisation.TensorNet import QtreeTensorNet
    from qtensor.optimisation.late_parallelisation import LateParOptimizer

    out = {'generator': 'tests/golden/make_slicing_golden.py', 'cases': []}
    for n, gseed, p, aseed, n_edges in CASES:
        G = graphs.regular(n, seed=gseed)
        gamma, beta = graphs.angles(p, aseed)
        for edge in list(G.edges())[:n_edges]:
            comp = DefaultQAOAComposer(G, gamma=gamma, beta=beta)
            comp.energy_expectation_lightcone(edge)
            circuit = comp.circuit
            order_opt = OrderingOptimizer()
            order_opt.optimize(QtreeTensorNet.from_qtree_gates(circuit))
            width = int(order_opt.treewidth)
            for drop in (2, 3):
                tn = QtreeTensorNet.from_qtree_gates(circuit)
                ignored = set(int(v) for v in tn.ket_vars + tn.bra_vars)
                opt = LateParOptimizer(target_tw=width - drop)
                schedule = opt.optimize(tn)
                order = [int(x) for prefix, _ in schedule for x in prefix]
                sliced = [int(x) for _, sv in schedule for x in sv if int(x) not in ignored]
                out['cases'].append({'nodes': n, 'graph_seed': gseed, 'p': p, 'angle_seed': aseed,
                                     'edge': [int(edge[0]), int(edge[1])], 'width': width,
                                     'target_tw': width - drop, 'late_width': int(opt.treewidth),
                                     'order': order, 'sliced': sliced})
                print(n, p, edge, 'width', width, 'target', width - drop, 'sliced', sliced, flush=True)
    with open(os.path.join(HERE, 'late_slicing_reference.json'), 'w') as f:
        json.dump(out, f, separators=(',', ':'))


if __name__ == '__main__':
    main()
