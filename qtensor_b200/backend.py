"""Drop-in bucket backend: QTensor's ``BucketBackend`` API on the GPU.

``B200Backend`` implements the three methods of ``BucketBackend``
(qtensor/ProcessingFrameworks.py:13-21) with the semantics of
``NumpyBackend`` (:23-37, arithmetic restated in-repo by
``CMKLExtendedBackend.process_bucket`` :45-147), so
``QtreeSimulator(bucket_backend=B200Backend())`` and
``QAOAQtreeSimulator(composer, bucket_backend=B200Backend())`` run unchanged:

* ``get_sliced_buckets`` sorts every tensor's indices by ``int``, transposes
  and slices its array (integer slices drop the axis, ``slice`` objects keep
  it) and uploads all arrays in one host-to-device copy as complex64;
* ``process_bucket`` launches ``qtb_bucket_c64`` (K1): the product of the
  bucket's tensors over the sorted union of their indices, summed over the
  first (bucket) index unless ``no_sum``; the result is a new tensor of the
  caller's tensor class named ``E<first index>`` (``Ef`` for scalars);
* ``get_result_data`` returns the result as a numpy array.

Indices of size 1 (sliced bra/ket variables) take part in the index
bookkeeping but not in the arithmetic; sizes other than 1 and 2 raise.
The backend pickles without its device state (lazy CUDA initialisation), so
``energy_expectation_parallel`` worker processes each open their own context.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check


class B200Backend:
    """QTensor ``BucketBackend`` running every bucket as one sm_100a kernel."""

    def __init__(self, device=None):
        self._device_index = device
        self._device = None
        self._lib = None

    # -- lazy device state (not pickled)
    def __getstate__(self):
        return {'_device_index': self._device_index}

    def __setstate__(self, state):
        self._device_index = state['_device_index']
        self._device = None
        self._lib = None

    def _ensure(self):
        if self._device is None:
            if not torch.cuda.is_available():
                raise RuntimeError('B200Backend needs a CUDA device; there is no CPU fallback')
            idx = torch.cuda.current_device() if self._device_index is None else self._device_index
            self._lib = _lib.lib()
            check(self._lib.qtb_init(idx))
            self._device = torch.device('cuda', idx)
        return self._device

    # ------------------------------------------------------------ slicing
    def get_sliced_buckets(self, buckets, data_dict, slice_dict):
        device = self._ensure()
        pending = []            # (bucket_idx, tensor, indices, host array)
        for b, bucket in enumerate(buckets):
            for tensor in bucket:
                order = sorted(range(len(tensor.indices)), key=lambda i: int(tensor.indices[i]))
                data = tensor.data if tensor.data is not None else data_dict[tensor.data_key]
                if isinstance(data, torch.Tensor):
                    data = data.detach().cpu().numpy()
                data = np.transpose(np.asarray(data), order)
                indices = [tensor.indices[i] for i in order]
                bounds = tuple(slice_dict.get(v, slice(None)) for v in indices)
                data = data[bounds]
                kept = [v for v, s in zip(indices, bounds) if not isinstance(s, (int, np.integer))]
                kept = [v.copy(size=n) if v.size != n else v for v, n in zip(kept, data.shape)]
                pending.append((b, tensor, kept, np.ascontiguousarray(data, dtype=np.complex64)))
        sizes = [a.size for *_, a in pending]
        flat = np.empty(max(1, sum(sizes)), dtype=np.complex64)
        pos = 0
        for (*_, a), n in zip(pending, sizes):
            flat[pos:pos + n] = a.reshape(-1)
            pos += n
        dev = torch.from_numpy(flat).pin_memory().to(device, non_blocking=True)
        out = [[] for _ in buckets]
        pos = 0
        for (b, tensor, kept, a), n in zip(pending, sizes):
            view = dev[pos:pos + n].view(a.shape)
            pos += n
            out[b].append(tensor.copy(indices=tuple(kept), data=view))
        return out

    # ------------------------------------------------------------ buckets
    def _as_device(self, tensor):
        data = tensor.data
        if not isinstance(data, torch.Tensor):
            data = torch.from_numpy(np.ascontiguousarray(np.asarray(data), dtype=np.complex64))
        data = data.to(self._device, dtype=torch.complex64)
        order = sorted(range(len(tensor.indices)), key=lambda i: int(tensor.indices[i]))
        if order != list(range(len(order))):
            data = data.permute(order)
        indices = [tensor.indices[i] for i in order]
        return indices, data.contiguous()

    def process_bucket(self, bucket, no_sum=False):
        self._ensure()
        if len(bucket) == 0:
            raise ValueError('process_bucket: empty bucket')
        if len(bucket) > _lib.QTB_MAX_BUCKET_INPUTS:
            raise ValueError('process_bucket: more than {} tensors in a bucket'.format(
                _lib.QTB_MAX_BUCKET_INPUTS))
        operands = [self._as_device(t) for t in bucket]
        union = {}
        for indices, _ in operands:
            for v in indices:
                union.setdefault(int(v), v)
        union = [union[k] for k in sorted(union)]
        for v in union:
            if v.size not in (1, 2):
                raise NotImplementedError('index {} has size {}; only binary (and sliced, size-1) '
                                          'indices are supported'.format(v, v.size))
        live = [v for v in union if v.size == 2]
        pos = {int(v): i for i, v in enumerate(live)}
        u = len(live)
        if u > _lib.QTB_MAX_BUCKET_VARS:
            raise ValueError('process_bucket: {} variables exceed the kernel limit'.format(u))
        summed = (not no_sum) and len(union) > 0
        sum_first = 1 if summed and union[0].size == 2 else 0
        out_indices = tuple(union[1:]) if summed else tuple(union)
        desc = _lib.BucketDesc()
        desc.n_inputs = len(operands)
        desc.n_vars = u
        desc.sum_first = sum_first
        ptrs = (ctypes.c_void_p * len(operands))()
        for t, (indices, data) in enumerate(operands):
            m = 0
            for v in indices:
                if v.size == 2:
                    m |= 1 << (u - 1 - pos[int(v)])
            desc.masks[t] = m
            ptrs[t] = data.data_ptr()
        out = torch.empty([v.size for v in out_indices], dtype=torch.complex64, device=self._device)
        stream = torch.cuda.current_stream(self._device).cuda_stream
        check(self._lib.qtb_bucket_c64(ctypes.byref(desc), ptrs, ctypes.c_void_p(out.data_ptr()),
                                       ctypes.c_void_p(stream)))
        tag = union[0].identity if union else 'f'
        return type(bucket[0])('E{}'.format(tag), out_indices, data=out)

    def get_result_data(self, result):
        data = result.data
        if isinstance(data, torch.Tensor):
            return data.cpu().numpy()
        return np.asarray(data)
