"""Drop-in ``B200Backend`` (K1 bucket kernel through the C ABI) against the
oracle's NumpyBackend: single buckets and whole simulations."""
import numpy as np
import pytest
import torch

import qtensor_port as port
from conftest import golden_graph
from qtree import np_framework
from qtree.optimizer import Tensor, Var

pytestmark = pytest.mark.gpu

TOL = 1e-5   # complex64 plain path vs complex128 oracle, absolute on |values| <= 1


def _backend():
    from qtensor_b200.backend import B200Backend
    return B200Backend()


def _random_bucket(rng, n_vars, k, sliced=()):
    """k tensors over subsets of n_vars binary variables, all containing var 0."""
    vars_ = [Var(i, size=1 if i in sliced else 2) for i in range(n_vars)]
    bucket = []
    for _ in range(k):
        others = [v for v in vars_[1:] if rng.random() < 0.5]
        idx = [vars_[0]] + others
        shape = [v.size for v in idx]
        data = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        bucket.append(Tensor('T', idx, data=data))
    return bucket


def _to_backend(backend, bucket):
    data_dict = {}
    tensors = []
    for i, t in enumerate(bucket):
        data_dict[('t', i)] = t.data
        tensors.append(Tensor(t.name, t.indices, data_key=('t', i)))
    return backend.get_sliced_buckets([tensors], data_dict, {})[0]


@pytest.mark.parametrize('n_vars,k', [(1, 1), (2, 2), (3, 1), (5, 3), (8, 4), (12, 6), (18, 3),
                                      (22, 2)])
@pytest.mark.parametrize('no_sum', [False, True])
def test_process_bucket_matches_numpy(cuda_device, n_vars, k, no_sum):
    rng = np.random.default_rng(n_vars * 31 + k)
    bucket = _random_bucket(rng, n_vars, k)
    ref = np_framework.process_bucket_np(bucket, no_sum=no_sum)
    backend = _backend()
    out = backend.process_bucket(_to_backend(backend, bucket), no_sum=no_sum)
    assert [int(v) for v in out.indices] == [int(v) for v in ref.indices]
    assert out.name == ref.name
    got = backend.get_result_data(out)
    scale = max(1.0, np.max(np.abs(ref.data)))
    assert np.max(np.abs(got - ref.data)) < 1e-5 * scale * k


def test_process_bucket_sliced_and_scalar(cuda_device):
    rng = np.random.default_rng(7)
    bucket = _random_bucket(rng, 6, 3, sliced=(0, 3))
    ref = np_framework.process_bucket_np(bucket)
    backend = _backend()
    out = backend.process_bucket(_to_backend(backend, bucket))
    assert [int(v) for v in out.indices] == [int(v) for v in ref.indices]
    assert np.allclose(backend.get_result_data(out), ref.data, atol=1e-4)
    scalars = [Tensor('s', (), data=np.array(0.5 + 0.25j)), Tensor('s', (), data=np.array(2.0))]
    out = backend.process_bucket(_to_backend(backend, scalars))
    assert out.name == 'Ef' and out.indices == ()
    assert abs(complex(backend.get_result_data(out)) - (1.0 + 0.5j)) < 1e-6


def test_process_bucket_unsorted_input(cuda_device):
    rng = np.random.default_rng(3)
    a, b, c = Var(0), Var(1), Var(2)
    data = rng.standard_normal((2, 2, 2)) + 0j
    t_sorted = Tensor('t', (a, b, c), data=data)
    t_perm = Tensor('t', (c, a, b), data=np.transpose(data, (2, 0, 1)).copy())
    backend = _backend()
    for t in (t_perm,):
        out = backend.process_bucket([Tensor('t', t.indices, data=torch.from_numpy(t.data))])
        ref = np_framework.process_bucket_np([t_sorted])
        assert np.allclose(backend.get_result_data(out), ref.data, atol=1e-5)


def test_process_bucket_rejects_unsupported(cuda_device):
    backend = _backend()
    big = Var(0, size=3)
    with pytest.raises(NotImplementedError):
        backend.process_bucket([Tensor('t', (big,), data=np.ones(3))])
    with pytest.raises(ValueError):
        backend.process_bucket([Tensor('t', (Var(0),), data=np.ones(2))] * 17)


@pytest.mark.parametrize('comp', ['default', 'cx', 'zz'])
def test_simulator_with_b200_backend_cfg1(cuda_device, comp):
    """QTensor's simulator path (port) with the drop-in backend: every edge
    term within 1e-5 of the reference, energy within 1e-5 relative."""
    G, w = golden_graph('cfg1_' + comp)
    backend = _backend()
    total = 0
    for k, edge in enumerate(G.edges()):
        circ = port.lightcone_circuit(G, edge, w['gamma'], w['beta'], comp)
        amp = port.simulate_amplitude(circ, backend=backend)
        assert abs(amp[0] - complex(*w['terms'][k])) < TOL
        total += amp[0]
    E = port.post_process_energy(G, total)
    assert abs(E - w['energy']) <= 1e-5 * abs(w['energy'])


def test_backend_pickles_without_device_state():
    import pickle
    from qtensor_b200.backend import B200Backend
    b = pickle.loads(pickle.dumps(B200Backend(device=0)))
    assert b._device is None and b._device_index == 0


def test_perf_backend_times_every_bucket(cuda_device, capsys):
    """PerfB200Backend (the reference's PerfBackend around the drop-in
    backend): same amplitudes, one device time per distinct bucket, the
    reference's ideal flop count, and the text report with its totals."""
    from qtensor_b200.backend import B200Backend, PerfB200Backend, PerfBackend
    G, w = golden_graph('cfg1_default')
    edge = list(G.edges())[0]
    circ = port.lightcone_circuit(G, edge, w['gamma'], w['beta'], 'default')
    perf = PerfB200Backend()
    amp = port.simulate_amplitude(circ, backend=perf)
    assert abs(amp[0] - complex(*w['terms'][0])) < TOL
    results = perf.profile_results
    assert results and all(t > 0 for _, t in results.values())
    rep = perf.gen_report()
    assert 'Total bucket contractions: {}'.format(len(results)) in rep
    assert '| max |' in capsys.readouterr().out
    wrapped = PerfBackend.from_backend(B200Backend)
    assert isinstance(wrapped.backend, B200Backend)
    # union of 3 indices -> result 2^2, two tensors -> 4 * (1 + 2)
    a, b, c = Var(1), Var(2), Var(3)
    assert PerfBackend._perfect_bucket_flop([(a, b), (a, c)]) == 12
