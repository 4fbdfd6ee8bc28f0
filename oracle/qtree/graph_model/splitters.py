"""Tree-trimming slicing (``Optimizer.py:203-205``) is not part of the oracle."""


def split_graph_by_tree_trimming(graph, n_var_parallel):
    raise NotImplementedError('tree-trimming slicing is not restated in the oracle')


def split_graph_by_tree_trimming_width(graph, n_var_parallel):
    raise NotImplementedError('tree-trimming slicing is not restated in the oracle')
