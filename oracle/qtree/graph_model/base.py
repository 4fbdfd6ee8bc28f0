"""Line graph of a bucket network and elimination bookkeeping.

Oracle restatement (test infrastructure only).  The line graph is a networkx
``MultiGraph`` whose nodes are ``int(var)`` with attributes ``name`` and
``size`` (read by ``qtensor/optimisation/Optimizer.py:55-56``); each tensor adds
a clique over its non-ignored variables, a single-variable tensor a self loop.
Nodes are inserted in order of first appearance over buckets, tensors and
indices, which fixes the tie-breaking of the greedy orderer
(``qtensor/utils.py:23-32`` takes the first minimum in node order).
"""
import itertools

import networkx as nx


def buckets2graph(buckets, ignore_variables=()):
    ignore = set(ignore_variables)
    graph = nx.MultiGraph()
    for bucket in buckets:
        for tensor in bucket:
            nodes = [v for v in tensor.indices if v not in ignore]
            for v in nodes:
                if int(v) not in graph:
                    graph.add_node(int(v), name=v.name, size=v.size)
            ids = [int(v) for v in nodes]
            if len(ids) > 1:
                graph.add_edges_from(itertools.combinations(ids, 2), tensor=tensor.name)
            elif len(ids) == 1:
                graph.add_edge(ids[0], ids[0], tensor=tensor.name)
    return graph


def make_clique_on(graph, nodes):
    """Copy of ``graph`` with the given variables made mutually adjacent."""
    ids = [int(v) for v in nodes]
    g = graph.copy()
    g.add_edges_from(itertools.combinations(ids, 2))
    return g


def get_equivalent_peo(graph, peo, clique_vertices):
    """Move the clique (free) variables to the end of ``peo``; eliminating a
    clique last does not change the width of a perfect elimination order."""
    clique = [int(v) for v in clique_vertices]
    head = [v for v in peo if int(v) not in clique]
    tail_lookup = {int(v): v for v in peo if int(v) in clique}
    tail = [tail_lookup.get(c, c) for c in clique]
    return head + tail


def relabel_graph_nodes(graph, label_dict):
    """Relabel ``graph`` by ``label_dict`` (old -> new); returns the new graph
    and the inverse mapping (new -> old), as ``Optimizer.py:199-206`` expects."""
    g = nx.relabel_nodes(graph, label_dict, copy=True)
    inverse = {new: old for old, new in label_dict.items()}
    return g, inverse


def eliminate_node(graph, node):
    """Remove ``node`` and connect its neighbours into a clique (in place)."""
    nbrs = set(graph[node]) - {node}
    graph.remove_node(node)
    if len(nbrs) > 1:
        graph.add_edges_from(itertools.combinations(sorted(nbrs), 2))


def remove_node(graph, node):
    """Remove ``node`` without fill-in: slicing a variable deletes it."""
    graph.remove_node(node)


def get_treewidth_from_peo(graph, peo):
    """Largest neighbour count met while eliminating ``peo`` in order."""
    g = nx.Graph(graph)
    g.remove_edges_from(list(nx.selfloop_edges(g)))
    width = 0
    for v in peo:
        v = int(v)
        if v not in g:
            continue
        width = max(width, len(g[v]))
        eliminate_node(g, v)
    return width


def get_contraction_costs(graph):
    """Memory (elements) and flops of eliminating the nodes in ``int`` order:
    each step builds a tensor over the node and its neighbours."""
    g = nx.Graph(graph)
    g.remove_edges_from(list(nx.selfloop_edges(g)))
    mems, flops = [], []
    for v in sorted(g.nodes, key=int):
        nbrs = list(g[v])
        size = 2 ** len(nbrs)
        mems.append(size)
        flops.append(2 * size * max(1, g.degree(v)))
        eliminate_node(g, v)
    return mems, flops
