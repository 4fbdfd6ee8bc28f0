"""The drop-in claim, checked against the reference's own driver.

The reference's ``QAOAQtreeSimulator`` with its ``NumpyBackend`` was run
through a recorder (``tests/golden/make_dropin_trace.py``); every call its
driver made into the backend -- ``get_sliced_buckets``, each
``process_bucket(bucket, no_sum)`` of ``bucket_elimination``,
``get_result_data`` -- is replayed here into ``B200Backend`` in the same order
with the same arguments.  Every result must carry the reference's name and
indices, and its data must match the recorded NumpyBackend result within the
complex64 tolerance: in full for results of up to 16 elements, else by its
sum and squared norm; every edge's amplitude must match the recorded one.
"""
import numpy as np
import pytest

import dropin_replay

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.mark.parametrize('name', ['cfg1', 'cfg2'])
def test_reference_driver_calls_replay_on_b200_backend(cuda_device, name):
    import torch
    from qtensor_b200.backend import B200Backend
    w = dropin_replay.load()[name]
    be = B200Backend()
    n_calls = 0
    for rec in w['edges']:
        def check(k, res, rec=rec):
            call = rec['calls'][k]
            assert res.name == call['name']
            assert [dropin_replay.var_rec(v) for v in res.indices] == call['indices']
            data = res.data
            assert isinstance(data, torch.Tensor) and data.is_cuda   # stays on the device
            got = data.detach().cpu().numpy().astype(np.complex128).reshape(-1)
            if 'data' in call:
                ref = np.array([complex(*z) for z in call['data']])
                assert got.shape == ref.shape
                assert np.max(np.abs(got - ref)) < TOL
            else:
                scale = max(1.0, np.sqrt(call['norm2']))
                assert abs(got.sum() - complex(*call['sum'][0])) < TOL * scale * np.sqrt(got.size)
                assert abs(np.sum(np.abs(got) ** 2) - call['norm2']) < TOL * max(1.0, call['norm2'])
        amp, results = dropin_replay.replay_edge(be, rec, check=check)
        n_calls += len(results)
        ref = np.array([complex(*z) for z in rec['amplitude']])
        assert amp.shape == ref.shape and np.max(np.abs(amp - ref)) < TOL
    assert n_calls == sum(len(r['calls']) for r in w['edges'])


def test_replayed_amplitudes_sum_to_reference_energy_cfg1(cuda_device):
    """All 30 edges of the N=20 p=1 workload through the replay give the
    reference's energy (qtensor/QAOASimulator.py:27-41) within 1e-5."""
    from conftest import golden
    from qtensor_b200.backend import B200Backend
    w = dropin_replay.load()['cfg1']
    be = B200Backend()
    total = sum(dropin_replay.replay_edge(be, rec)[0][0] for rec in w['edges'])
    E = (len(w['graph_edges']) - total.real) / 2
    E_ref = golden()['cfg1_default']['energy']
    assert abs(E - E_ref) <= TOL * abs(E_ref)
