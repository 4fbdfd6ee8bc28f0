"""Index helpers: slicing dictionaries and einsum expressions.

Oracle restatement of the ``qtree.utils`` helpers used by
``qtensor/Simulate.py:55-56`` and ``qtensor/FeynmanSimulator.py:23``.
Test infrastructure only.
"""
import string

import numpy as np

_ALPHABET = string.ascii_letters


def num_to_alpha(n):
    """Einsum letter for a small index number (52 letters, enough for one bucket)."""
    if n >= len(_ALPHABET):
        raise ValueError('einsum index {} out of range'.format(n))
    return _ALPHABET[n]


def get_einsum_expr(idx1, idx2):
    """``'ab,bc->abc'``-style expression multiplying two index lists into
    their sorted union (no summation)."""
    union = sorted(set(idx1) | set(idx2))
    rank = {v: i for i, v in enumerate(union)}
    a = ''.join(num_to_alpha(rank[v]) for v in idx1)
    b = ''.join(num_to_alpha(rank[v]) for v in idx2)
    c = ''.join(num_to_alpha(rank[v]) for v in union)
    return '{},{}->{}'.format(a, b, c)


def unravel_index(value, dimensions):
    """Mixed-radix digits of ``value``, most significant first (numpy order)."""
    if len(dimensions) == 0:
        return ()
    return tuple(int(x) for x in np.unravel_index(int(value), tuple(dimensions)))


def slice_from_bits(value, variables):
    """``{var: slice(b, b+1)}`` fixing ``variables`` to the digits of ``value``."""
    digits = unravel_index(value, [v.size for v in variables])
    return {v: slice(d, d + 1) for v, d in zip(variables, digits)}
