"""Line-graph helpers (``qtree.graph_model`` subset).

Oracle restatement, test infrastructure only; call sites:
``qtensor/optimisation/TensorNet.py:40,55``, ``Optimizer.py:37,73,82,155,199-209``,
``late_parallelisation.py:144,184,188``, ``utils.py:121``.
"""
from . import base
from . import splitters
from . import peo_calculation
from .base import (buckets2graph, make_clique_on, get_equivalent_peo,  # noqa: F401
                   relabel_graph_nodes, get_contraction_costs,
                   get_treewidth_from_peo, eliminate_node, remove_node)
