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
    """Mixed-radix digits of ``value``, most significant first (the order of
    ``numpy.unravel_index``, computed here for any number of dimensions:
    lightcones of more than 64 qubits exceed numpy's array rank)."""
    value = int(value)
    total = 1
    for d in dimensions:
        total *= int(d)
    if not 0 <= value < max(total, 1):
        raise ValueError('index {} out of range for dimensions {}'.format(value, tuple(dimensions)))
    digits = []
    for d in reversed(dimensions):
        value, r = divmod(value, int(d))
        digits.append(r)
    return tuple(reversed(digits))


def slice_from_bits(value, variables):
    """``{var: slice(b, b+1)}`` fixing ``variables`` to the digits of ``value``."""
    digits = unravel_index(value, [v.size for v in variables])
    return {v: slice(d, d + 1) for v, d in zip(variables, digits)}
