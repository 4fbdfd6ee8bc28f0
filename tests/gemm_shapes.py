"""GEMM structure of compiled plans (measurement infrastructure, CPU only).

For every bucket whose sum has exactly two arena operands A and B (masks a,
b over the union, the summed variable on top), weighted by the bucket's
product size 2^u:
  * min(M, N) = 2^min(|a \\ b|, |b \\ a|): the smaller side of the matrix
    product the bucket would be as a GEMM (shared kept variables are batch);
  * K = 2^chain: the summed variable plus the following ops that sum the
    result alone (no other arena operand), which could be merged into one
    contraction.
Tensor cores pay only when min(M, N) and K are large; the plans of the
N=1000 p=3, N=256 p=4 and Erdos-Renyi N=400 p=3 workloads are printed.

    python tests/gemm_shapes.py
"""
import collections
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, 'tests')]

import networkx as nx  # noqa: E402
import numpy as np  # noqa: E402

from conftest import golden_graph  # noqa: E402
from qtensor_b200 import _lib  # noqa: E402
from qtensor_b200.plan import NetworkPlan, graph_csr  # noqa: E402


def workloads():
    yield '3-regular N=1000 p=3', golden_graph('cfg3')[0], 3, 24
    yield '3-regular N=256 p=4', golden_graph('cfg4')[0], 4, 24
    yield 'Erdos-Renyi N=400 p=3', nx.erdos_renyi_graph(400, 3 / 399, seed=24323709), 3, 22


def shapes(plan):
    ex = plan.export()
    nets, ops, ins = ex['nets'], ex['ops'], ex['ins']
    side, chain_k = collections.Counter(), collections.Counter()
    total = 0.0
    for n in nets:
        L = [ops[int(n['op_begin']) + i] for i in range(int(n['n_ops']))]

        def arena_inputs(o):
            return [ins[int(o['in_begin']) + t] for t in range(int(o['k']))
                    if not int(ins[int(o['in_begin']) + t]['src']) & _lib.SRC_TABLE]
        for i, o in enumerate(L):
            ai = arena_inputs(o)
            if not o['sum'] or len(ai) != 2:
                continue
            size = 2.0 ** int(o['u'])
            total += size
            a, b = int(ai[0]['mask']), int(ai[1]['mask'])
            side[min(bin(a & ~b).count('1'), bin(b & ~a).count('1'))] += size
            dst, length = int(o['dst']), 1
            for q in L[i + 1:]:
                qa = arena_inputs(q)
                if any(int(d['src']) == dst for d in qa):
                    if q['sum'] and len(qa) == 1:
                        length += 1
                        dst = int(q['dst'])
                    else:
                        break
            chain_k[length] += size
    return side, chain_k, total


def main():
    for name, G, p, max_width in workloads():
        plan = NetworkPlan(2 * p)
        plan.set_order_trials(16)
        plan.set_max_width(max_width)
        plan.add_lightcones(graph_csr(G), np.array(list(G.edges())), p, 0, np.zeros(2 * p))
        side, chain_k, total = shapes(plan)
        print(name)
        print('  min(M, N) = 2^k, share of two-operand sums:',
              {k: round(v / total, 3) for k, v in sorted(side.items())})
        print('  merged K = 2^chain, share:', {2 ** k: round(v / total, 3) for k, v in sorted(chain_k.items())})


if __name__ == '__main__':
    main()
