"""Host-side logic that needs no GPU: serving admission control and the
loud failure of the product paths without a CUDA device."""
import pytest
import torch

from qtensor_b200.serve import AdmissionControl, Result


def test_admission_respects_budget_and_slots():
    adm = AdmissionControl(budget_bytes=100, slots=2)
    assert adm.fits_ever(100) and not adm.fits_ever(101)
    a = adm.try_admit(60)
    assert a == 0
    assert adm.try_admit(50) is None          # memory: 60 + 50 > 100
    b = adm.try_admit(40)
    assert b == 1
    assert adm.try_admit(1) is None           # no slot left
    adm.release(a, 60)
    assert adm.used == 40 and adm.try_admit(60) == 0
    adm.release(0, 60)
    adm.release(1, 40)
    assert adm.used == 0 and adm.free_slots == [0, 1]


def test_result_timeline_splits_latency():
    r = Result(-1.5, 3, 4, submitted=10.0, admitted=10.25, finished=10.75, compiled=10.125)
    assert r.compile_s == pytest.approx(0.125)
    assert r.wait_s == pytest.approx(0.125)
    assert r.gpu_s == pytest.approx(0.5)
    assert r.compile_s + r.wait_s + r.gpu_s == pytest.approx(r.latency)
    # without a compile stamp the wait is counted as compile time
    r = Result(0.0, 0, 0, 1.0, 2.0, 2.0)
    assert r.wait_s == 0.0 and r.compile_s == pytest.approx(1.0)


def test_engine_needs_cuda_loudly(monkeypatch):
    from qtensor_b200 import engine
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: False)
    with pytest.raises(RuntimeError, match='no CPU fallback'):
        engine.QAOAEnergyEngine()


def test_server_needs_cuda_loudly(monkeypatch):
    from qtensor_b200 import serve
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: False)
    with pytest.raises(RuntimeError, match='no CPU fallback'):
        serve.QAOAServer()


def test_backend_needs_cuda_loudly(monkeypatch):
    from qtensor_b200.backend import B200Backend
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: False)
    with pytest.raises(RuntimeError, match='no CPU fallback'):
        B200Backend().get_sliced_buckets([[]], {}, {})


def test_composer_names_follow_the_reference():
    from qtensor_b200.qaoa import composer_name

    class DefaultQAOAComposer:
        pass

    class ZZQtreeQAOAComposer:
        pass

    assert composer_name(DefaultQAOAComposer) == 'default'
    assert composer_name(ZZQtreeQAOAComposer) == 'zz'
    assert composer_name('cx') == 'cx'
    with pytest.raises(ValueError):
        composer_name('qiskit')


def test_simulators_need_cuda_loudly(monkeypatch):
    from qtensor_b200 import simulator, qaoa
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: False)
    with pytest.raises(RuntimeError, match='no CPU fallback'):
        simulator.QtreeSimulator()
    with pytest.raises(RuntimeError, match='no CPU fallback'):
        qaoa.QAOAQtreeSimulator()


def test_perf_backend_needs_cuda_loudly(monkeypatch):
    from qtensor_b200.backend import PerfB200Backend
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: False)
    with pytest.raises(RuntimeError, match='CUDA'):
        PerfB200Backend().process_bucket([object()])


def test_edge_subset_digest_is_memoised_for_tuples_only():
    """The plan-cache key of an edge subset: a tuple passed again is not
    rehashed (a rank's shard), a list is hashed every call (it may change in
    place), and equal subsets give equal keys."""
    import hashlib
    import types
    from qtensor_b200.engine import QAOAEnergyEngine
    fake = types.SimpleNamespace(_edge_digests={})
    shard = (0, 2, 4, 6)
    t1, d1 = QAOAEnergyEngine._edges_digest(fake, shard)
    assert t1 == shard and d1 == hashlib.sha1(repr(shard).encode()).hexdigest()
    assert id(shard) in fake._edge_digests
    t2, d2 = QAOAEnergyEngine._edges_digest(fake, shard)
    assert (t2, d2) == (t1, d1)
    as_list = [0, 2, 4, 6]
    t3, d3 = QAOAEnergyEngine._edges_digest(fake, as_list)
    assert (t3, d3) == (t1, d1) and id(as_list) not in fake._edge_digests
    as_list.append(8)
    assert QAOAEnergyEngine._edges_digest(fake, as_list)[1] != d1
