"""GEMM structure of compiled plans, asserted on the CPU.

For every bucket whose sum has exactly two arena operands A and B (masks a,
b over the union, the summed variable on top), weighted by the bucket's
product size 2^u:
  * min(M, N) = 2^min(|a \\ b|, |b \\ a|): the smaller side of the matrix
    product the bucket would be as a GEMM (shared kept variables are batch);
  * K = 2^chain: the summed variable plus the following ops that sum the
    result alone (no other arena operand), which could be merged into one
    contraction.
Tensor cores pay only when min(M, N) and K are large.
"""
import collections

import numpy as np

import graphs
from conftest import golden_graph
from qtensor_b200 import _lib
from qtensor_b200.plan import NetworkPlan, graph_csr


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


def _plan(G, p):
    plan = NetworkPlan(2 * p)
    plan.set_order_trials(16)
    plan.set_max_width(29, 1024)
    plan.add_lightcones(graph_csr(G), np.array(list(G.edges())), p, 0, np.zeros(2 * p))
    return plan


def _share(counter, total, pred):
    return sum(v for k, v in counter.items() if pred(k)) / total


def test_headline_plans_have_no_gemm_structure():
    """3-regular N=1000 p=3 and N=256 p=4: every two-operand sum is an
    outer or Hadamard product (the smaller side at most 2^4 for all but a
    sliver of the work), and chains that could merge into one contraction
    reach K >= 32 for under 0.1 % (N=1000 p=3) and 5 % (N=256 p=4) of it:
    a tensor-core tile would be padding, so these products stay on the CUDA
    cores."""
    for name, limit_side, limit_k in (('cfg3', 0.99, 0.001), ('cfg4', 0.95, 0.05)):
        G = golden_graph(name)[0]
        side, chain_k, total = shapes(_plan(G, 4 if name == 'cfg4' else 3))
        assert _share(side, total, lambda k: k <= 4) >= limit_side, name
        assert _share(chain_k, total, lambda k: 2 ** k >= 32) <= limit_k, name


def test_deeper_circuits_start_to_show_gemm_structure():
    """At p=5 (3-regular N=256, beyond the configured workloads) the sides
    grow: most two-operand work has min(M, N) >= 32, and a few percent of
    it merges to K >= 32."""
    G = graphs.regular(256)
    side, chain_k, total = shapes(_plan(G, 5))
    assert _share(side, total, lambda k: k >= 5) >= 0.4
    assert _share(chain_k, total, lambda k: 2 ** k >= 32) >= 0.03
