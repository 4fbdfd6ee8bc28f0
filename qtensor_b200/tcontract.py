"""The reference's ``tcontract`` module on the GPU.

``CMKLExtendedBackend`` (qtensor/ProcessingFrameworks.py:41-147) imports a
native module ``tcontract`` (lazily, qtensor/tools/lazy_import/__init__.py:41)
that the reference does not ship.  Its two calls, with the reference's
argument order and in-place output:

* ``mkl_contract_complex(a, b, c)``: ``c[n,m,k] = a[n,m] * b[n,k]``
  (ProcessingFrameworks.py:65-66);
* ``mkl_contract_sum(a, b, c)``: ``C[f,m,n] = sum_k A[k,f,m] * B[k,f,n]``
  (:129-130);

on CUDA complex64 torch tensors, through ``qtb_contract_outer_c64`` and
``qtb_contract_sum_c64``.  The contract-sum runs on the tcgen05 tensor cores
in 3xTF32 with FP32 accumulation when its summed dimension is large
(``mode``: 0 automatic, 1 CUDA cores, 2 tensor cores).  There is no CPU
path: arguments must be CUDA tensors.
"""
import ctypes

import torch

from . import _lib

MODES = {'auto': 0, 'simt': 1, 'tensor': 2}


def _check_tensor(x, name, dims):
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise TypeError('{} must be a CUDA tensor (there is no CPU path)'.format(name))
    if x.dtype != torch.complex64:
        raise TypeError('{} must be complex64, not {}'.format(name, x.dtype))
    if x.dim() != dims:
        raise ValueError('{} must have {} dimensions, not {}'.format(name, dims, x.dim()))
    if not x.is_contiguous():
        raise ValueError('{} must be contiguous'.format(name))


def _stream(x):
    return ctypes.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)


def mkl_contract_complex(a, b, c):
    """``c[n,m,k] = a[n,m] * b[n,k]`` (in place into ``c``)."""
    _check_tensor(a, 'a', 2)
    _check_tensor(b, 'b', 2)
    _check_tensor(c, 'c', 3)
    n, m = a.shape
    k = b.shape[1]
    if b.shape[0] != n or tuple(c.shape) != (n, m, k):
        raise ValueError('shapes {}, {}, {} do not match c[n,m,k] = a[n,m] b[n,k]'.format(
            tuple(a.shape), tuple(b.shape), tuple(c.shape)))
    lib = _lib.lib()
    _lib.check(lib.qtb_contract_outer_c64(a.data_ptr(), b.data_ptr(), c.data_ptr(), n, m, k, _stream(a)))
    return c


def contract_sum_scratch_bytes(K, F, M, N, mode='auto'):
    n = ctypes.c_size_t()
    _lib.check(_lib.lib().qtb_contract_sum_scratch_bytes(K, F, M, N, MODES[mode], ctypes.byref(n)))
    return n.value


def mkl_contract_sum(a, b, c, mode='auto', scratch=None):
    """``C[f,m,n] = sum_k A[k,f,m] * B[k,f,n]`` (in place into ``c``).
    ``scratch`` (uint8 CUDA tensor of ``contract_sum_scratch_bytes``) is
    allocated when not given; its first int32 is the kernel's status word."""
    _check_tensor(a, 'a', 3)
    _check_tensor(b, 'b', 3)
    _check_tensor(c, 'c', 3)
    K, F, M = a.shape
    N = b.shape[2]
    if tuple(b.shape[:2]) != (K, F) or tuple(c.shape) != (F, M, N):
        raise ValueError('shapes {}, {}, {} do not match C[f,m,n] = sum_k A[k,f,m] B[k,f,n]'.format(
            tuple(a.shape), tuple(b.shape), tuple(c.shape)))
    need = contract_sum_scratch_bytes(K, F, M, N, mode)
    if scratch is None:
        scratch = torch.empty(need, dtype=torch.uint8, device=a.device)
    elif scratch.numel() * scratch.element_size() < need:
        raise ValueError('scratch of {} bytes, {} needed'.format(scratch.numel() * scratch.element_size(), need))
    lib = _lib.lib()
    _lib.check(lib.qtb_contract_sum_c64(a.data_ptr(), b.data_ptr(), c.data_ptr(), K, F, M, N, MODES[mode],
                                        scratch.data_ptr(), scratch.numel() * scratch.element_size(),
                                        _stream(a)))
    return c
