"""The reference's ``tcontract`` products on the GPU (qtb_contract_*_c64) and
``B200ExtendedBackend``, the counterpart of ``CMKLExtendedBackend``
(qtensor/ProcessingFrameworks.py:41-147), against complex128 numpy.

The contract-sum ``C[f,m,n] = sum_k A[k,f,m] B[k,f,n]`` is checked on the
tcgen05 tensor-core path (3xTF32 products, FP32 accumulation) and on the
CUDA-core path, on shapes that fill whole 128 x 128 x 32 tiles and on
ragged ones that are padded; the bar is 1e-5 of the largest output
magnitude."""
import numpy as np
import pytest

import dropin_replay

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _rand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)


def _sum_ref(A, B):
    return np.einsum('kfm,kfn->fmn', A, B)


@pytest.mark.parametrize('mode', ['tensor', 'simt', 'auto'])
@pytest.mark.parametrize('K,F,M,N', [(32, 1, 128, 128), (64, 2, 256, 128), (40, 3, 200, 72),
                                     (256, 1, 128, 384), (2, 3, 5, 7), (1, 1, 1, 1), (1000, 1, 130, 129)])
def test_contract_sum_matches_complex128(cuda_device, mode, K, F, M, N):
    import torch
    from qtensor_b200 import tcontract
    rng = np.random.default_rng(K * 7 + M)
    A, B = _rand(rng, (K, F, M)), _rand(rng, (K, F, N))
    a = torch.from_numpy(A.astype(np.complex64)).to(cuda_device)
    b = torch.from_numpy(B.astype(np.complex64)).to(cuda_device)
    c = torch.full((F, M, N), complex(np.nan, np.nan), dtype=torch.complex64, device=cuda_device)
    scratch = torch.empty(tcontract.contract_sum_scratch_bytes(K, F, M, N, mode), dtype=torch.uint8,
                          device=cuda_device)
    tcontract.mkl_contract_sum(a, b, c, mode=mode, scratch=scratch)
    torch.cuda.synchronize()
    assert int(scratch[:4].view(torch.int32).item()) == 0        # no bounded wait gave up
    got = c.cpu().numpy().astype(np.complex128)
    ref = _sum_ref(A.astype(np.complex64).astype(np.complex128), B.astype(np.complex64).astype(np.complex128))
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - ref)) <= TOL * np.max(np.abs(ref))


def test_tensor_core_and_cuda_core_paths_agree(cuda_device):
    """Both paths sum in FP32; 3xTF32 products keep the tensor-core result
    within FP32 rounding of the CUDA-core one."""
    import torch
    from qtensor_b200 import tcontract
    rng = np.random.default_rng(5)
    K, F, M, N = 512, 2, 256, 256
    a = torch.from_numpy(_rand(rng, (K, F, M)).astype(np.complex64)).to(cuda_device)
    b = torch.from_numpy(_rand(rng, (K, F, N)).astype(np.complex64)).to(cuda_device)
    ct = torch.empty((F, M, N), dtype=torch.complex64, device=cuda_device)
    cs = torch.empty_like(ct)
    tcontract.mkl_contract_sum(a, b, ct, mode='tensor')
    tcontract.mkl_contract_sum(a, b, cs, mode='simt')
    torch.cuda.synchronize()
    d = (ct - cs).abs().max().item()
    assert d <= 1e-5 * cs.abs().max().item()


def test_contract_outer_matches_numpy(cuda_device):
    import torch
    from qtensor_b200 import tcontract
    rng = np.random.default_rng(3)
    for n, m, k in ((4, 8, 2), (1, 1, 1), (32, 16, 64)):
        A, B = _rand(rng, (n, m)), _rand(rng, (n, k))
        a = torch.from_numpy(A.astype(np.complex64)).to(cuda_device)
        b = torch.from_numpy(B.astype(np.complex64)).to(cuda_device)
        c = torch.empty((n, m, k), dtype=torch.complex64, device=cuda_device)
        tcontract.mkl_contract_complex(a, b, c)
        ref = np.einsum('nm,nk->nmk', A, B)
        assert np.max(np.abs(c.cpu().numpy() - ref)) < 1e-6


def test_contract_rejects_bad_shapes_and_host_tensors(cuda_device):
    import torch
    from qtensor_b200 import tcontract
    a = torch.zeros((2, 1, 4), dtype=torch.complex64, device=cuda_device)
    b = torch.zeros((2, 1, 3), dtype=torch.complex64, device=cuda_device)
    with pytest.raises(ValueError):
        tcontract.mkl_contract_sum(a, b, torch.zeros((1, 4, 4), dtype=torch.complex64, device=cuda_device))
    with pytest.raises(TypeError):
        tcontract.mkl_contract_sum(a.cpu(), b, torch.zeros((1, 4, 3), dtype=torch.complex64))


@pytest.mark.parametrize('mode', ['auto', 'tensor'])
@pytest.mark.parametrize('name', ['cfg1', 'cfg2'])
def test_extended_backend_replays_reference_driver(cuda_device, name, mode):
    """The reference driver's recorded backend calls through
    B200ExtendedBackend (mode 'tensor' sends every contract-sum of the
    buckets to the tcgen05 path): every amplitude matches the recorded
    NumpyBackend value within 1e-5, and so does every intermediate result
    on the CUDA-core path.  On the tensor-core path an intermediate may sit
    up to 5e-5 (relative squared norm) from the recorded one: each 3xTF32
    contraction is within about 2^-22 of complex64 (the dropped lo x lo
    term, round-toward-zero inside a k block), and a network chains about
    130 of them before its scalar result."""
    from qtensor_b200.backend import B200ExtendedBackend
    w = dropin_replay.load()[name]
    be = B200ExtendedBackend(mode=mode)
    mid_tol = TOL if mode != 'tensor' else 5 * TOL
    for rec in w['edges']:
        def check(k, res, rec=rec):
            call = rec['calls'][k]
            assert res.name == call['name']
            assert [dropin_replay.var_rec(v) for v in res.indices] == call['indices']
            got = res.data.detach().cpu().numpy().astype(np.complex128).reshape(-1)
            if 'data' in call:
                assert np.max(np.abs(got - [complex(*z) for z in call['data']])) < mid_tol
            else:
                assert abs(np.sum(np.abs(got) ** 2) - call['norm2']) < mid_tol * max(1.0, call['norm2'])
        amp, _ = dropin_replay.replay_edge(be, rec, check=check)
        assert np.max(np.abs(amp - [complex(*z) for z in rec['amplitude']])) < TOL
