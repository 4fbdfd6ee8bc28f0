"""Record the reference's own calls into its bucket backend, for replay on the GPU.

Runs the reference package's ``QAOAQtreeSimulator`` (imported from a
read-only reference checkout through ``oracle/refimport.py``, on the oracle
``qtree``) with a recording subclass of the reference's own ``NumpyBackend``
(qtensor/ProcessingFrameworks.py:23-37) as its ``bucket_backend``.  The
reference's driver -- ``QAOASimulator._get_edge_energy`` -> ``simulate`` ->
``QtreeSimulator.simulate_batch`` (qtensor/Simulate.py:66-94) ->
``TensorNet.slice`` -> ``backend.get_sliced_buckets`` ->
``bucket_elimination(..., backend.process_bucket)`` -> ``get_result_data`` --
makes every call; the recorder writes down, per edge:

* the buckets given to ``get_sliced_buckets`` (tensor names, indices as
  (identity, size, name), their data arrays (deduplicated) and the slice
  dict (integers, or slice bounds);
* every ``process_bucket(bucket, no_sum)`` call in order, its bucket as
  references to sliced input tensors or to earlier results, and the
  NumpyBackend result: name, indices, data (in full up to 16 elements, else
  its sum and squared norm);
* the amplitude ``get_result_data`` returned.

``tests/test_gpu_dropin.py`` replays the calls into ``B200Backend`` on a GPU
box, which has no reference checkout.

    python tests/golden/make_dropin_trace.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
sys.path.insert(0, os.path.join(ROOT, 'tests'))

import graphs  # noqa: E402
from refimport import import_reference  # noqa: E402

FULL_DATA_LIMIT = 16
WORKLOADS = [
    # name, graph, p, angle seed, composer, edges recorded
    ('cfg1', lambda: graphs.regular(20), 1, 0, 'default', None),
    ('cfg2', lambda: graphs.regular(100), 3, 0, 'default', 8),
]


def cplx_list(a):
    """Complex values as [re, im] pairs, 10 significant digits (the replay
    compares complex64 results at 1e-5)."""
    a = np.asarray(a, dtype=np.complex128).reshape(-1)
    return [[float('%.10g' % z.real), float('%.10g' % z.imag)] for z in a]


def var_rec(v):
    return [int(v.identity), int(v.size), str(v.name)]


def main():
    qtensor = import_reference()
    if qtensor is None:
        sys.exit('no reference checkout found (set QTENSOR_REFERENCE)')
    from qtensor import QAOAQtreeSimulator, DefaultQAOAComposer
    from qtensor.ProcessingFrameworks import NumpyBackend

    class RecordingBackend(NumpyBackend):
        """The reference's NumpyBackend, writing down what its caller asks."""

        def start(self):
            self.edge = {'buckets': [], 'slice': [], 'calls': []}
            self.arrays = {}        # bytes -> index into self.array_list
            self.array_list = []
            self.origin = {}        # id(tensor) -> reference in the trace
            self.keep = []          # tensors kept alive while their ids are in use

        def _array(self, data):
            a = np.ascontiguousarray(np.asarray(data, dtype=np.complex128))
            blob = a.tobytes() + repr(a.shape).encode()
            if blob not in self.arrays:
                self.arrays[blob] = len(self.array_list)
                self.array_list.append({'shape': list(a.shape), 'data': cplx_list(a)})
            return self.arrays[blob]

        def get_sliced_buckets(self, buckets, data_dict, slice_dict):
            for bucket in buckets:
                recs = []
                for t in bucket:
                    data = t.data if t.data is not None else data_dict[t.data_key]
                    recs.append({'name': t.name, 'indices': [var_rec(v) for v in t.indices],
                                 'array': self._array(data)})
                self.edge['buckets'].append(recs)
            # an integer drops the axis, a slice keeps it (start, stop, step)
            self.edge['slice'] = [[var_rec(v), int(s) if isinstance(s, (int, np.integer))
                                   else [s.start, s.stop, s.step]] for v, s in slice_dict.items()]
            sliced = super().get_sliced_buckets(buckets, data_dict, slice_dict)
            for b, bucket in enumerate(sliced):
                for j, t in enumerate(bucket):
                    self.origin[id(t)] = ['s', b, j]
                    self.keep.append(t)
            return sliced

        def process_bucket(self, bucket, no_sum=False):
            refs = [self.origin[id(t)] for t in bucket]
            res = super().process_bucket(bucket, no_sum=no_sum)
            data = np.asarray(res.data, dtype=np.complex128)
            call = {'in': refs, 'no_sum': bool(no_sum), 'name': res.name,
                    'indices': [var_rec(v) for v in res.indices],
                    'sum': cplx_list(data.sum()), 'norm2': float(np.sum(np.abs(data) ** 2))}
            if data.size <= FULL_DATA_LIMIT:
                call['data'] = cplx_list(data)
            self.origin[id(res)] = ['r', len(self.edge['calls'])]
            self.keep.append(res)
            self.edge['calls'].append(call)
            return res

        def get_result_data(self, result):
            out = super().get_result_data(result)
            self.edge['amplitude'] = cplx_list(np.asarray(out).reshape(-1))
            return out

    out = {'generator': 'tests/golden/make_dropin_trace.py', 'workloads': {}}
    for name, make_graph, p, seed, comp, n_edges in WORKLOADS:
        G = make_graph()
        gamma, beta = graphs.angles(p, seed)
        backend = RecordingBackend()
        sim = QAOAQtreeSimulator(DefaultQAOAComposer, bucket_backend=backend)
        edges = list(G.edges())[:n_edges] if n_edges else list(G.edges())
        recs = []
        for edge in edges:
            backend.start()
            amp = sim._get_edge_energy(G, gamma, beta, edge)
            rec = backend.edge
            rec['edge'] = [int(edge[0]), int(edge[1])]
            rec['arrays'] = backend.array_list
            assert np.allclose(np.asarray(amp).reshape(-1), [complex(*rec['amplitude'][0])])
            recs.append(rec)
        out['workloads'][name] = {'graph_nodes': G.number_of_nodes(), 'p': p, 'gamma': gamma,
                                  'beta': beta, 'composer': comp, 'edges': recs,
                                  'graph_edges': [list(e) for e in G.edges()]}
        print('{}: {} edges, {} process_bucket calls'.format(
            name, len(recs), sum(len(r['calls']) for r in recs)), flush=True)
    with open(os.path.join(HERE, 'dropin_trace.json'), 'w') as f:
        json.dump(out, f, separators=(',', ':'))


if __name__ == '__main__':
    main()
