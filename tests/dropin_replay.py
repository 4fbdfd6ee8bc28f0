"""Replay the reference's recorded backend calls into ``B200Backend``.

``tests/golden/dropin_trace.json`` (made by ``make_dropin_trace.py`` from the
reference's own ``QAOAQtreeSimulator`` with a recording ``NumpyBackend``)
holds, per edge, the buckets the reference's driver gave
``get_sliced_buckets``, then every ``process_bucket(bucket, no_sum)`` call it
made (qtensor/Simulate.py:90-94 through ``bucket_elimination``) and every
result.  ``replay_edge`` makes the same calls, in the same order, on a
backend: sliced inputs and earlier results are passed exactly as the
reference passed them, scalar results are multiplied in call order (as
``bucket_elimination`` does) and ``get_result_data`` returns the amplitude.
The tensors are ``Tensor``/``Var`` below: the interface of qtree's classes
that the reference's driver hands a backend (qtree itself is not needed).
"""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TRACE = os.path.join(HERE, 'golden', 'dropin_trace.json')


class Var:
    """A contraction index as qtree's ``Var``: ``int(v)`` is its identity,
    with ``.size``, ``.name`` and ``copy``."""
    __slots__ = ('identity', 'size', 'name')

    def __init__(self, identity, size=2, name=None):
        self.identity = int(identity)
        self.size = int(size)
        self.name = name if name is not None else 'v_{}'.format(identity)

    def copy(self, identity=None, size=None, name=None):
        if identity is None:
            identity = self.identity
            name = self.name if name is None else name
        return Var(identity, self.size if size is None else size, name)

    def __int__(self):
        return self.identity

    __index__ = __int__

    def __hash__(self):
        return hash((self.identity, self.name, self.size))

    def __eq__(self, other):
        return (isinstance(other, Var) and (self.identity, self.size, self.name)
                == (other.identity, other.size, other.name))

    def __lt__(self, other):
        return self.identity < int(other)

    def __repr__(self):
        return self.name


class Tensor:
    """A named tensor as qtree's ``Tensor``: indices, and ``data`` or a
    ``data_key`` into the caller's data dict."""

    def __init__(self, name, indices, data_key=None, data=None):
        self.name = name
        self.indices = tuple(indices)
        self.data_key = data_key
        self.data = data

    def copy(self, name=None, indices=None, data_key=None, data=None):
        return Tensor(self.name if name is None else name,
                      self.indices if indices is None else indices,
                      self.data_key if data_key is None else data_key,
                      self.data if data is None else data)


def load():
    with open(TRACE) as f:
        return json.load(f)['workloads']


def _var(rec):
    return Var(rec[0], size=rec[1], name=rec[2])


def var_rec(v):
    return [int(v.identity), int(v.size), str(v.name)]


def edge_inputs(rec):
    """The unsliced buckets, data dict and slice dict of one recorded edge."""
    arrays = [np.array([complex(*z) for z in a['data']], dtype=np.complex128).reshape(a['shape'])
              for a in rec['arrays']]
    buckets = [[Tensor(t['name'], [_var(v) for v in t['indices']], data_key=('trace', t['array']))
                for t in bucket] for bucket in rec['buckets']]
    data_dict = {('trace', i): a for i, a in enumerate(arrays)}
    slice_dict = {_var(v): (s if isinstance(s, int) else slice(*s)) for v, s in rec['slice']}
    return buckets, data_dict, slice_dict


def replay_edge(backend, rec, inputs=None, check=None):
    """Make the recorded calls on ``backend``; returns the amplitude (numpy
    array) and the results of every ``process_bucket`` call.  ``check(k,
    result)`` is called after call k when given."""
    buckets, data_dict, slice_dict = inputs if inputs is not None else edge_inputs(rec)
    sliced = backend.get_sliced_buckets(buckets, data_dict, slice_dict)
    results, scalar = [], None
    for k, call in enumerate(rec['calls']):
        bucket = [sliced[r[1]][r[2]] if r[0] == 's' else results[r[1]] for r in call['in']]
        res = backend.process_bucket(bucket, no_sum=call['no_sum'])
        if check is not None:
            check(k, res)
        results.append(res)
        if len(res.indices) == 0:
            scalar = res.data if scalar is None else scalar * res.data
    amp = backend.get_result_data(Tensor('result', (), data=scalar))
    return np.asarray(amp).reshape(-1), results
