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


class B200ExtendedBackend(B200Backend):
    """QTensor's ``CMKLExtendedBackend`` (qtensor/ProcessingFrameworks.py:41-147)
    on the GPU, its absent native ``tcontract`` module replaced by
    ``qtensor_b200.tcontract``: the bucket's first tensors are merged by
    outer products over their common indices (``mkl_contract_complex``), the
    last one is contracted with a sum over the bucket index
    (``mkl_contract_sum``, on the tensor cores when its shape is large;
    ``mode`` forces 'simt' or 'tensor').  Inputs are sliced and uploaded as
    by ``B200Backend``; index bookkeeping, transposes and result names follow
    the reference's, so results equal ``NumpyBackend``'s within complex64
    rounding (3xTF32 on the tensor cores).  A single-tensor sum goes through
    ``qtb_bucket_c64`` as in ``B200Backend``."""

    def __init__(self, device=None, mode='auto'):
        super().__init__(device)
        self.mode = mode

    def __getstate__(self):
        state = super().__getstate__()
        state['mode'] = self.mode
        return state

    def __setstate__(self, state):
        super().__setstate__(state)
        self.mode = state.get('mode', 'auto')

    def _data(self, tensor):
        data = tensor.data
        if not isinstance(data, torch.Tensor):
            data = torch.from_numpy(np.ascontiguousarray(np.asarray(data), dtype=np.complex64))
        return data.to(self._device, dtype=torch.complex64)

    @staticmethod
    def _size(indices, data, ix):
        return data.shape[list(indices).index(ix)]

    def _merge(self, result_data, result_indices, tensor):
        """``merge_with_result`` (:50-78): c[n,m,k] = a[n,m] b[n,k] over the
        common (n), result-only (m) and tensor-only (k) indices."""
        from . import tcontract
        ixa, ixb = tuple(result_indices), tuple(tensor.indices)
        b_data = self._data(tensor)
        common = sorted(set(ixa) & set(ixb), key=int)
        dist_a = [x for x in ixa if x not in common]
        dist_b = [x for x in ixb if x not in common]
        a = result_data.permute([ixa.index(x) for x in common + dist_a]).contiguous()
        b = b_data.permute([ixb.index(x) for x in common + dist_b]).contiguous()
        n = int(np.prod([self._size(ixa, result_data, x) for x in common], dtype=np.int64))
        m = int(np.prod([self._size(ixa, result_data, x) for x in dist_a], dtype=np.int64))
        k = int(np.prod([self._size(ixb, b_data, x) for x in dist_b], dtype=np.int64))
        c = torch.empty((n, m, k), dtype=torch.complex64, device=self._device)
        tcontract.mkl_contract_complex(a.reshape(n, m), b.reshape(n, k), c)
        out_indices = tuple(sorted(set(ixa + ixb), key=int))
        ixc = common + dist_a + dist_b
        sizes = [self._size(ixa, result_data, x) if x in ixa else self._size(ixb, b_data, x) for x in ixc]
        out = c.reshape(sizes).permute([ixc.index(x) for x in out_indices])
        return out.contiguous(), out_indices

    def process_bucket(self, bucket, no_sum=False):
        from . import tcontract
        self._ensure()
        if len(bucket) == 0:
            raise ValueError('process_bucket: empty bucket')
        if len(bucket) < 2 and not no_sum:
            return super().process_bucket(bucket, no_sum=no_sum)
        result_indices = tuple(bucket[0].indices)
        result_data = self._data(bucket[0])
        for tensor in bucket[1:-1]:
            result_data, result_indices = self._merge(result_data, result_indices, tensor)
        tag = result_indices[0].identity if result_indices else 'f'
        make = type(bucket[0])
        if no_sum:
            if len(bucket) > 1:
                result_data, result_indices = self._merge(result_data, result_indices, bucket[-1])
            return make('E{}'.format(tag), result_indices, data=result_data)
        # contraction with the sum over the bucket index (:112-147)
        last = bucket[-1]
        last_data = self._data(last)
        ixa, ixb = result_indices, tuple(last.indices)
        k, fm, fn = ixa[:1], ixa[1:], ixb[1:]
        if ixb[:1] != k:
            raise ValueError('process_bucket: the last tensor does not start with the bucket index')
        f = tuple(sorted(set(fm) & set(fn), key=int))
        m = tuple(x for x in fm if x not in f)
        n = tuple(x for x in fn if x not in f)
        a = result_data.permute([ixa.index(x) for x in k + f + m]).contiguous()
        b = last_data.permute([ixb.index(x) for x in k + f + n]).contiguous()
        shapes = {x: self._size(ixb, last_data, x) for x in ixb}
        shapes.update({x: self._size(ixa, result_data, x) for x in ixa})
        K, F, M, N = [int(np.prod([shapes[x] for x in grp], dtype=np.int64)) for grp in (k, f, m, n)]
        c = torch.empty((F, M, N), dtype=torch.complex64, device=self._device)
        tcontract.mkl_contract_sum(a.reshape(K, F, M), b.reshape(K, F, N), c, mode=self.mode)
        out_indices = tuple(sorted(set(ixa + ixb), key=int))[1:]
        ixc = f + m + n
        out = c.reshape([shapes[x] for x in ixc]).permute([ixc.index(x) for x in out_indices])
        return make('E{}'.format(tag), out_indices, data=out.contiguous())


class PerfBackend:
    """Per-bucket timing around another backend, the counterpart of
    QTensor's ``PerfBackend`` (qtensor/ProcessingFrameworks.py:152-234).

    ``Backend`` is the wrapped class (``B200Backend`` by default;
    ``from_backend`` builds a subclass for another one).  Every
    ``process_bucket`` is bracketed by CUDA events on the current stream, so
    the recorded time is the bucket's device time, not its launch time;
    events are resolved when a report is asked for.  Records are keyed by
    ``str`` of the bucket's index tuples, as the reference keys them.
    ``gen_report`` returns the reference's text report (the slowest
    buckets, then totals) and prints a markdown table of per-bucket figures
    with their max / mean / sum."""
    Backend = B200Backend

    def __init__(self, *args, print=False, num_lines=20, **kwargs):
        self.backend = self.Backend(*args, **kwargs)
        self._print = print
        self.max_lines = num_lines
        self._pending = {}           # key -> (indices, start event, end event)
        self._profile_results = {}   # key -> (indices, seconds)

    @classmethod
    def from_backend(cls, backend, *args, **kwargs):
        """A ``PerfBackend`` around ``backend`` (a backend class)."""
        class CustomGeneratedBackend(cls):
            Backend = backend
        return CustomGeneratedBackend(*args, **kwargs)

    def process_bucket(self, bucket, no_sum=False):
        if not torch.cuda.is_available():
            raise RuntimeError('PerfBackend times buckets with CUDA events and needs a CUDA device')
        indices = [tensor.indices for tensor in bucket]
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record()
        result = self.backend.process_bucket(bucket, no_sum=no_sum)
        end.record()
        self._pending[str(indices)] = (indices, start, end)
        return result

    def get_sliced_buckets(self, buckets, data_dict, slice_dict):
        return self.backend.get_sliced_buckets(buckets, data_dict, slice_dict)

    def get_result_data(self, result):
        return self.backend.get_result_data(result)

    @property
    def profile_results(self):
        """``{key: (indices, seconds)}`` of every bucket timed so far."""
        for key, (indices, start, end) in self._pending.items():
            end.synchronize()
            seconds = start.elapsed_time(end) / 1e3
            if self._print:
                print('PROF:: perf data process bucket time: {}'.format(seconds))
            self._profile_results[key] = (indices, seconds)
        self._pending.clear()
        return self._profile_results

    @staticmethod
    def _perfect_bucket_flop(bucket_indices):
        """Ideal operation count of a bucket, the reference's estimate
        (ProcessingFrameworks.py:186-196): result size (the union less the
        contracted index) times (one summation + one multiplication per
        tensor)."""
        union = set().union(*[set(ixs) for ixs in bucket_indices])
        size_of_result = 2 ** (len(union) - 1) if union else 1
        return size_of_result * (1 + len(bucket_indices))

    def gen_report(self):
        data = sorted(self.profile_results.values(), key=lambda pair: pair[1], reverse=True)
        max_lines = self.max_lines
        lines = [str([i, ixs, t]) for i, (ixs, t) in enumerate(data[:max_lines])]
        rep = '\n'.join(lines)
        if len(data) > max_lines:
            rep += '\n ... and {} lines more...'.format(len(data) - max_lines)
        fields = ('bucket_len', 'time', 'flop', 'FLOPS', 'max_size', 'min_size', 'result_size')
        records = []
        for ixs, t in data[:max_lines]:
            flop = self._perfect_bucket_flop(ixs)
            records.append((len(ixs), t, flop, flop / t if t > 0 else float('inf'),
                            max(len(i) for i in ixs), min(len(i) for i in ixs),
                            len(set().union(*[set(i) for i in ixs])) - 1))
        if records:
            table = ['| measure | ' + ' | '.join(fields) + ' |', '|---' * (len(fields) + 1) + '|']
            cols = list(zip(*records))
            for name, fn in (('max', max), ('mean', lambda c: sum(c) / len(c)), ('sum', sum)):
                table.append('| {} | '.format(name) + ' | '.join('{:.4g}'.format(fn(c)) for c in cols) + ' |')
            print('\n'.join(table))
        total_time = sum(t for _, t in data)
        rep += '\n======\n'
        rep += 'Total time: ' + str(total_time)
        rep += '\nTotal bucket contractions: ' + str(len(data))
        rep += '\nMean time for contraction: ' + str(total_time / len(data) if data else 0.0)
        rep += '\n'
        return rep


class PerfB200Backend(PerfBackend):
    """``PerfBackend`` around ``B200Backend`` (the reference's
    ``PerfNumpyBackend`` pattern)."""
    Backend = B200Backend
