"""NumPy bucket processing -- the arithmetic of QTensor's ``NumpyBackend``.

Oracle restatement (test infrastructure only) of
``qtree.np_framework.process_bucket_np`` / ``get_sliced_np_buckets`` as called
by ``qtensor/ProcessingFrameworks.py:29-34``.  The semantics follow the
in-repo restatement ``CMKLExtendedBackend.process_bucket``
(``qtensor/ProcessingFrameworks.py:45-147``) and the einsum form of
``scratchpad/node_parallel/node_parallel.py:50-64``:

* the running result starts as ``bucket[0]``; each further tensor is
  multiplied in by an einsum whose output indices are the union of both
  index sets sorted by ``int`` (``ProcessingFrameworks.py:69-72``);
* unless ``no_sum``, axis 0 (the smallest variable -- the bucket variable) is
  summed out and dropped (``ProcessingFrameworks.py:100-103,132-146``);
* the result is named ``E<identity of the first index>`` or ``Ef`` for a
  scalar (``ProcessingFrameworks.py:86-89``).
"""
import numpy as np

from .optimizer import Tensor
from .utils import get_einsum_expr


def get_sliced_np_buckets(buckets, data_dict, slice_dict):
    """Attach arrays to every tensor and apply ``slice_dict``.

    Each tensor's indices are sorted by ``int`` and its array transposed to
    match; a ``slice`` entry keeps the axis (with the new size), an integer
    entry removes it (``qtensor/FeynmanSimulator.py:18-25`` passes integers,
    ``qtensor/Simulate.py:54-58`` passes ``slice_from_bits`` slices).
    """
    sliced_buckets = []
    for bucket in buckets:
        out = []
        for tensor in bucket:
            order = sorted(range(len(tensor.indices)), key=lambda i: int(tensor.indices[i]))
            data = data_dict[tensor.data_key] if tensor.data is None else tensor.data
            data = np.transpose(np.asarray(data), order)
            indices = [tensor.indices[i] for i in order]
            bounds = tuple(slice_dict.get(v, slice(None)) for v in indices)
            data = data[bounds]
            kept = [v for v, b in zip(indices, bounds) if not isinstance(b, (int, np.integer))]
            assert len(kept) == data.ndim, 'slicing dropped the wrong axes'
            kept = [v.copy(size=s) if v.size != s else v for v, s in zip(kept, data.shape)]
            out.append(tensor.copy(indices=kept, data=data))
        sliced_buckets.append(out)
    return sliced_buckets


def process_bucket_np(bucket, no_sum=False):
    """Multiply the tensors of ``bucket`` and sum over its first variable."""
    result_indices = tuple(bucket[0].indices)
    result_data = bucket[0].data
    for tensor in bucket[1:]:
        expr = get_einsum_expr([int(v) for v in result_indices],
                               [int(v) for v in tensor.indices])
        result_data = np.einsum(expr, result_data, tensor.data)
        result_indices = tuple(sorted(set(result_indices + tuple(tensor.indices)), key=int))

    if len(result_indices) > 0:
        tag = result_indices[0].identity
    else:
        tag = 'f'
    if no_sum or len(result_indices) == 0:
        return Tensor('E{}'.format(tag), result_indices, data=result_data)
    return Tensor('E{}'.format(tag), result_indices[1:], data=np.sum(result_data, axis=0))
