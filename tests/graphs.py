"""Seeded graphs and angles of the QAOA workloads used by tests, fixtures and
the benchmark.  The graphs are rebuilt with the same networkx calls every
time, so their node and adjacency order (which fixes the reference's cone
qubit numbering) is reproducible on any machine with the same networkx."""
import networkx as nx
import numpy as np

PETERSEN_EDGES = [[0, 1], [1, 2], [2, 3], [3, 4], [4, 0], [0, 5], [1, 6], [2, 7], [3, 8],
                  [4, 9], [5, 7], [5, 8], [6, 8], [6, 9], [7, 9]]


def regular(n, d=3, seed=0):
    return nx.random_regular_graph(d, n, seed=seed)


def angles(p, seed=0):
    """gamma, beta ~ U[0, pi)^p from ``numpy.random.default_rng(seed)``."""
    rng = np.random.default_rng(seed)
    return list(rng.uniform(0, np.pi, p)), list(rng.uniform(0, np.pi, p))


def family(kind, n, d):
    """The graph families of qtensor/tests/test_qaoa_energy.py:16-43 (seeded)."""
    if kind == 'random':
        return nx.random_regular_graph(d, n, seed=1)
    if kind == 'grid2d':
        return nx.convert_node_labels_to_integers(nx.grid_2d_graph(n, n))
    if kind == 'line':
        G = nx.Graph()
        G.add_edges_from(zip(range(n - 1), range(1, n)))
        return G
    raise ValueError(kind)


def petersen():
    G = nx.Graph()
    G.add_edges_from(PETERSEN_EDGES)
    return G


def by_name(name):
    """Rebuild the graph of a golden workload by its fixture name."""
    if name.startswith('cfg1'):
        return regular(20)
    if name == 'cfg2':
        return regular(100)
    if name == 'cfg3':
        return regular(1000)
    if name == 'cfg4':
        return regular(256)
    if name == 'petersen_p9':
        return petersen()
    if name.startswith('test_'):
        _, kind, n, p, d = name.split('_')
        return family(kind, int(n[1:]), int(d[1:]))
    raise KeyError(name)


def erdos_renyi(n, seed, mean_degree=3):
    """Erdos-Renyi graph of the serving workload (edge probability mean_degree / (n - 1))."""
    return nx.erdos_renyi_graph(n, mean_degree / (n - 1), seed=seed)


# Graphs of the serving workload whose widest edges are the corner cases of
# the compiler (seeds as the serving stream draws them).
ER_P4_N109 = dict(n=109, seed=716218221, p=4)   # edges of width 40+: intractable
ER_P3_N335 = dict(n=335, seed=949594894, p=3)   # one edge of width 28-31
ER_P3_N213 = dict(n=213, seed=796350419, p=3)   # edges of width 28-31
