"""Continuous-batching server: every result equals the reference energy, is
the same alone and in a mix of concurrent requests, and a failing request
fails alone."""
import networkx as nx
import numpy as np
import pytest

import graphs
import qtensor_port as port
from conftest import golden_graph

pytestmark = pytest.mark.gpu


def _requests(n, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        N = int(rng.integers(16, 60))
        p = int(rng.integers(1, 4))
        if i % 2:
            G = nx.erdos_renyi_graph(N, 3 / (N - 1), seed=int(rng.integers(1 << 30)))
        else:
            G = nx.random_regular_graph(3, N + (N % 2), seed=int(rng.integers(1 << 30)))
        gamma, beta = graphs.angles(p, seed=int(rng.integers(1 << 30)))
        if G.number_of_edges():
            out.append((G, gamma, beta))
    return out


def test_server_matches_reference(cuda_device):
    from qtensor_b200.serve import QAOAServer
    G, w = golden_graph('cfg2')
    with QAOAServer() as srv:
        res = srv.submit(G, w['gamma'], w['beta']).result(timeout=120)
    assert abs(res.energy - w['energy']) <= 1e-5 * abs(w['energy'])
    assert res.edges == G.number_of_edges() and res.latency > 0
    assert res.submitted <= res.compiled <= res.admitted <= res.finished


def _wide_requests():
    """Two wide requests of the serving stream: Erdos-Renyi N=400 p=3, whose
    networks too large for shared memory run on the cluster executor when
    QTB_CLUSTER_MAX_ELEMS allows it, and Erdos-Renyi N=335 p=3 (seed
    949594894), whose widest edge (width 28, arenas of about 5 GB) runs in
    whole-GPU waves."""
    er400 = nx.erdos_renyi_graph(400, 3 / 399, seed=24323709)
    er335 = graphs.erdos_renyi(graphs.ER_P3_N335['n'], graphs.ER_P3_N335['seed'])
    return [(er400,) + tuple(graphs.angles(3, seed=1)), (er335,) + tuple(graphs.angles(3, seed=2))]


def test_alone_and_in_the_mix_agree(cuda_device, monkeypatch):
    """Each request's energy is identical whether it runs alone (one stream,
    one request at a time) or together with the others (four streams, all
    submitted at once), and equals the oracle's.  The mix holds small
    requests and two wide ones (cluster executor and wide waves), whose
    kernels overlap the others'."""
    from qtensor_b200.serve import QAOAServer
    monkeypatch.setenv('QTB_CLUSTER_MAX_ELEMS', str(1 << 22))
    reqs = _requests(14)
    reqs = reqs[:7] + _wide_requests() + reqs[7:]
    with QAOAServer(n_streams=1) as srv:
        alone = [srv.submit(*r).result(timeout=300) for r in reqs]
    with QAOAServer(n_streams=4) as srv:
        futs = [srv.submit(*r) for r in reqs]
        mixed = [f.result(timeout=300) for f in futs]
    assert [r.energy for r in alone] == [r.energy for r in mixed]
    assert max(r.networks for r in mixed) > 0
    for (G, gamma, beta), r in list(zip(reqs, mixed))[:4]:
        ref = float(port.energy_expectation(G, gamma, beta)[0])
        assert abs(r.energy - ref) <= 1e-5 * max(1.0, abs(ref))


def test_wide_requests_run_on_the_wide_executors(cuda_device, monkeypatch):
    """The wide requests of the mix really use the cluster executor (K5) and
    the wide waves (K4): their plans' launch classes say so."""
    from qtensor_b200.engine import QAOAEnergyEngine
    monkeypatch.setenv('QTB_CLUSTER_MAX_ELEMS', str(1 << 22))
    eng = QAOAEnergyEngine(order_trials=4)
    flags = []
    for G, gamma, beta in _wide_requests():
        eng.energy_expectation(G, gamma, beta)
        cg = eng.compile(G, 3, gamma, beta)
        flags.append([c[3] for c in cg.plan.last_launch_config()])
    assert any(f & 64 for f in flags[0])
    assert any(f & 4 for f in flags[1])


def test_failing_request_fails_alone(cuda_device):
    from qtensor_b200.serve import QAOAServer
    reqs = _requests(4, seed=3)
    with QAOAServer(memory_budget=1 << 30) as srv:
        bad_angles = srv.submit(reqs[0][0], [0.1, 0.2], [0.3])          # p mismatch
        empty = srv.submit(nx.empty_graph(5), [0.1], [0.2])             # no edges: energy 0
        good = [srv.submit(*r) for r in reqs]
        with pytest.raises(ValueError):
            bad_angles.result(timeout=60)
        assert empty.result(timeout=60).energy == 0.0
        energies = [f.result(timeout=120).energy for f in good]
    for (G, gamma, beta), e in zip(reqs, energies):
        ref = float(port.energy_expectation(G, gamma, beta)[0])
        assert abs(e - ref) <= 1e-5 * max(1.0, abs(ref))


def test_over_budget_request_is_rejected(cuda_device):
    from qtensor_b200.serve import QAOAServer
    G = graphs.regular(200)
    with QAOAServer(memory_budget=1024) as srv:
        with pytest.raises(MemoryError):
            srv.submit(G, [0.1], [0.2]).result(timeout=60)
