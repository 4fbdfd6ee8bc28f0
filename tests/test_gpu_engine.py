"""Batched engine (gate-table kernel + whole-network executor + fp64 energy
reduction, through the C ABI) against the reference fixtures."""
import numpy as np
import pytest
import torch

import graphs
import statevector as sv
from conftest import golden_graph

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _engine(**kw):
    from qtensor_b200.engine import QAOAEnergyEngine
    return QAOAEnergyEngine(**kw)


def _check(engine, name):
    G, w = golden_graph(name)
    terms = engine.edge_terms(G, w['gamma'], w['beta'])
    ref = np.array([complex(*t) for t in w['terms']])
    assert np.max(np.abs(terms - ref)) < TOL, name
    E = engine.energy_expectation(G, w['gamma'], w['beta'])
    assert abs(E - w['energy']) <= TOL * abs(w['energy']), (E, w['energy'])
    return E


@pytest.mark.parametrize('comp', ['default', 'cx', 'zz'])
def test_engine_reference_order_cfg1(cuda_device, comp):
    _check(_engine(composer=comp, ordering='reference'), 'cfg1_' + comp)


@pytest.mark.parametrize('name', ['test_random_n4_p4_d3', 'test_random_n10_p5_d2',
                                  'test_random_n14_p1_d3', 'test_grid2d_n3_p3_d0',
                                  'test_line_n8_p4_d0', 'petersen_p9'])
def test_engine_families(cuda_device, name):
    E = _check(_engine(ordering='reference'), name)
    if name == 'petersen_p9':
        assert abs(E - 12.0) < 1e-2       # qtensor/tests/qiskit_qaoa_energy.py:123


@pytest.mark.parametrize('name', ['cfg2', 'cfg3', 'cfg4'])
def test_engine_native_order_large(cuda_device, name):
    _check(_engine(ordering='native'), name)


def test_engine_full_size_p1_closed_form(cuda_device):
    """Size-independent pin at the full N=1000 size: p=1 edge terms equal the
    closed-form expectation of every edge."""
    G = graphs.regular(1000)
    gamma, beta = graphs.angles(1, seed=5)
    terms = _engine().edge_terms(G, gamma, beta)
    exact = np.array([sv.qaoa_p1_edge_term(G, e, gamma[0], beta[0]) for e in G.edges()])
    assert np.max(np.abs(terms - exact)) < TOL


@pytest.mark.parametrize('name,p,seeds,stride', [('cfg3', 3, range(100, 105), 60),
                                                  ('cfg4', 4, range(400, 403), 48)])
def test_engine_benchmark_angle_sets_against_oracle(cuda_device, name, p, seeds, stride):
    """The angle sets the benchmark times (N=1000 p=3: seeds 100 + i; N=256
    p=4: seeds 400 + i), contracted on one cached plan: every sampled edge
    term equals the complex128 oracle port's (QAOASimulator._get_edge_energy
    restated), so the timed steps compute the reference's values and not
    only the fixture's angles do."""
    import qtensor_port as port
    G, _ = golden_graph(name)
    edges = list(G.edges())
    eng = _engine()
    for seed in seeds:
        gamma, beta = graphs.angles(p, seed=seed)
        terms = eng.edge_terms(G, gamma, beta)
        for k in range(0, len(edges), stride):
            ref = complex(port.edge_energy(G, gamma, beta, edges[k]))
            assert abs(terms[k] - ref) < TOL, (seed, edges[k], terms[k], ref)


def test_engine_plan_reuse_across_angles(cuda_device):
    """A cached plan with new angles equals a fresh compile with those angles."""
    G = graphs.regular(100)
    eng = _engine()
    g1, b1 = graphs.angles(3, seed=1)
    g2, b2 = graphs.angles(3, seed=2)
    eng.energy_expectation(G, g1, b1)
    reused = eng.edge_terms(G, g2, b2)
    fresh = _engine().edge_terms(G, g2, b2)
    assert np.array_equal(reused, fresh)
    assert len(eng._cache) == 1


def test_engine_graph_replay_matches_direct_launch(cuda_device):
    """energy_expectation replays a captured CUDA graph; interleaved angle
    sets give the energy of a direct launch + host fp64 sum every time."""
    G = graphs.regular(200, seed=2)
    eng = _engine()
    sets = [graphs.angles(2, seed=s) for s in (1, 2, 1, 3)]
    for gamma, beta in sets:
        E = eng.energy_expectation(G, gamma, beta)
        terms = eng.edge_terms(G, gamma, beta).astype(np.complex128)
        direct = (G.number_of_edges() - np.sum(terms.real)) / 2
        assert abs(E - direct) < 1e-9 * G.number_of_edges()
    assert eng.energy_expectation(G, *sets[0]) == eng.energy_expectation(G, *sets[2])


def test_engine_deterministic_and_status_clean(cuda_device):
    G, w = golden_graph('cfg2')
    eng = _engine()
    a = eng.energy_expectation(G, w['gamma'], w['beta'])
    b = eng.energy_expectation(G, w['gamma'], w['beta'])
    assert a == b
    cg = eng.compile(G, 3, w['gamma'], w['beta'])
    assert cg.plan.device_status() == 0


def test_engine_rejects_bad_angles(cuda_device):
    with pytest.raises(ValueError):
        _engine().energy_expectation(graphs.regular(10), [0.1, 0.2], [0.3])


@pytest.mark.parametrize('name,max_width', [('cfg2', 9), ('cfg4', 17)])
def test_engine_sliced(cuda_device, name, max_width):
    """Sliced networks (2^k per edge, FeynmanSimulator semantics) give the
    reference's edge terms and energy."""
    eng = _engine(max_width=max_width)
    G, w = golden_graph(name)
    cg = eng.compile(G, len(w['gamma']), w['gamma'], w['beta'])
    assert cg.n_networks > cg.n_edges
    assert max(i['treewidth'] for i in cg.infos) < max_width
    _check(eng, name)


@pytest.mark.parametrize('slicing', ['tree_trim', 'late'])
@pytest.mark.parametrize('name,max_width', [('cfg2', 9), ('cfg4', 15)])
def test_engine_sliced_by_tree_trimming_and_late_slicing(cuda_device, name, max_width, slicing):
    """The TreeTrimSplitter and LateParOptimizer choices of sliced variables
    give the reference's edge terms and energy on the device."""
    eng = _engine(max_width=max_width, slicing=slicing)
    G, w = golden_graph(name)
    cg = eng.compile(G, len(w['gamma']), w['gamma'], w['beta'])
    assert cg.n_networks > cg.n_edges
    _check(eng, name)


def test_feynman_qaoa_with_tree_trim_splitter(cuda_device):
    """The reference's test_qaoa_energy_feynman (qtensor/tests/
    test_qaoa_energy.py:109-121): QtreeQAOAComposer on a 3-regular N=10
    graph at p=3, sliced by TreeTrimSplitter(max_tw=13, tw_bias=0) and by a
    tighter target, gives the plain energy; the oracle port agrees."""
    import qtensor_port as port
    G = graphs.regular(10, seed=1)
    gamma, beta = [np.pi / 3] * 3, [np.pi / 2] * 3
    plain = _engine(composer='cx', max_width=0).energy_expectation(G, gamma, beta)
    ref = float(port.energy_expectation(G, gamma, beta, 'cx')[0])
    assert abs(plain - ref) <= TOL * abs(ref)
    for target in (13, 8):
        eng = _engine(composer='cx', max_width=target + 1, slicing='tree_trim')
        assert abs(eng.energy_expectation(G, gamma, beta) - plain) <= TOL * abs(plain)
        eng = _engine(composer='cx', max_width=target + 1, slicing='late')
        assert abs(eng.energy_expectation(G, gamma, beta) - plain) <= TOL * abs(plain)


@pytest.mark.parametrize('name,max_width', [('cfg1_default', 24), ('cfg2', 24), ('cfg4', 24),
                                            ('cfg2', 9)])
def test_plain_path_matches_batched_and_reference(cuda_device, name, max_width):
    """The plain path (one bucket-kernel launch per bucket over the same
    compiled plans) gives the reference's edge terms and energy, and the
    batched executor's within complex64 rounding."""
    eng = _engine(max_width=max_width)
    G, w = golden_graph(name)
    plain = eng.edge_terms(G, w['gamma'], w['beta'], path='plain')
    batched = eng.edge_terms(G, w['gamma'], w['beta'])
    ref = np.array([complex(*t) for t in w['terms']])
    assert np.max(np.abs(plain - ref)) < TOL
    assert np.max(np.abs(plain - batched)) < TOL
    E = eng.energy_expectation(G, w['gamma'], w['beta'], path='plain')
    assert abs(E - w['energy']) <= TOL * abs(w['energy'])
    assert eng.compile(G, len(w['gamma']), w['gamma'], w['beta']).plan.device_status() == 0


@pytest.mark.parametrize('cluster_max,wide_batch', [(None, '3'), (None, '2'), (str(1 << 22), None)])
def test_wide_networks_match_plain_path(cuda_device, monkeypatch, cluster_max, wide_batch):
    """Erdos-Renyi N=400 p=3 (seed 24323709) with the reference's greedy rule
    alone (order_trials=0, slicing from width 22): 247 networks too large
    for shared memory (3.5 GB of arenas) run beside the shared-memory
    classes, by default in whole-GPU waves (K4), and with
    QTB_CLUSTER_MAX_ELEMS=2^22 as one thread-block cluster each when their
    arena is at most 32 MB (K5) and in waves above; the wave kernel with 8
    and with 4 elements per thread in flight (QTB_WIDE_BATCH); either way
    every edge term equals the plain per-bucket path's (an independent
    execution of the same plans) and the energies agree."""
    import networkx as nx
    if cluster_max is not None:
        monkeypatch.setenv('QTB_CLUSTER_MAX_ELEMS', cluster_max)
    if wide_batch is not None:                 # the wave kernel with 8 or 4 elements per thread
        monkeypatch.setenv('QTB_WIDE_BATCH', wide_batch)
    G = nx.erdos_renyi_graph(400, 3 / 399, seed=24323709)
    gamma, beta = graphs.angles(3, seed=1)
    eng = _engine(max_width=22, order_trials=0)
    batched = eng.edge_terms(G, gamma, beta)
    cg = eng.compile(G, 3, gamma, beta)
    cfg = cg.plan.last_launch_config()
    waves = [c for c in cfg if c[3] & 4]
    clusters = [c for c in cfg if c[3] & 64]
    if cluster_max is None:
        assert len(waves) >= 2 and not clusters
    else:
        assert clusters and clusters[0][0] >= 100
    plain = eng.edge_terms(G, gamma, beta, path='plain')
    assert np.max(np.abs(batched - plain)) < TOL
    E = eng.energy_expectation(G, gamma, beta)
    Ep = eng.energy_expectation(G, gamma, beta, path='plain')
    assert abs(E - Ep) <= TOL * abs(Ep)
    assert cg.plan.device_status() == 0


@pytest.mark.parametrize('schedule', ['classes', 'persistent:256', 'hybrid:512', 'hybrid:1024',
                                      'hybrid12:512', 'hybrid12:1024', 'warp:64', 'warp:128', 'warp:256'])
def test_every_schedule_matches_reference(cuda_device, monkeypatch, schedule):
    """Each executor schedule the autotuner may pick (size classes, one
    persistent queue, large-network classes + lean queue, large-network
    classes + warp-per-network queue, large-network classes + 96-thread lean
    queue at 12 CTAs per SM), forced through QTB_SCHEDULE, gives
    the reference's edge terms for all 1500 edges of the N=1000 p=3
    workload."""
    monkeypatch.setenv('QTB_SCHEDULE', schedule)
    eng = _engine()
    G, w = golden_graph('cfg3')
    terms = eng.edge_terms(G, w['gamma'], w['beta'])
    ref = np.array([complex(*t) for t in w['terms']])
    assert np.max(np.abs(terms - ref)) < TOL
    cfg = eng.compile(G, 3, w['gamma'], w['beta']).plan.last_launch_config()
    if schedule.startswith('hybrid12'):
        assert any(c[3] & 32 and c[1] == 96 for c in cfg)
    elif schedule.startswith('hybrid'):
        assert any(c[3] & 8 for c in cfg) and any(not c[3] & 2 for c in cfg)
    elif schedule.startswith('warp'):
        assert any(c[3] & 16 and c[1] == int(schedule[5:]) for c in cfg)
    elif schedule == 'classes':
        assert not any(c[3] & 2 for c in cfg)
    else:
        assert len(cfg) == 1 and cfg[0][3] & 2 and cfg[0][1] == 256


@pytest.mark.parametrize('schedule', ['persistent:128', 'hybrid:512', 'hybrid12:1024'])
def test_dynamic_claims_match_reference(cuda_device, monkeypatch, schedule):
    """Persistent launches that claim every network from their queue (the
    server's setting) give the same edge terms as the default, where a CTA
    starts on the job of its own index, and the reference's within TOL."""
    monkeypatch.setenv('QTB_SCHEDULE', schedule)
    G, w = golden_graph('cfg3')
    ref = np.array([complex(*t) for t in w['terms']])
    static = _engine().edge_terms(G, w['gamma'], w['beta'])
    dynamic = _engine(dynamic_claims=True).edge_terms(G, w['gamma'], w['beta'])
    assert np.max(np.abs(dynamic - ref)) < TOL
    assert np.array_equal(dynamic, static)   # same products in the same order


@pytest.mark.parametrize('name,p,max_width', [('cfg3', 3, 29), ('cfg4', 4, 29), ('cfg2', 3, 11)])
def test_element_records_match_blob_path(cuda_device, name, p, max_width):
    """The shared-memory executor contracting from element records gives the
    reference's edge terms, and the terms of the same plans decoded from
    their blobs (records off): N=1000 p=3, N=256 p=4, and N=100 p=3 sliced
    below its width."""
    G, w = golden_graph(name)
    ref = np.array([complex(*t) for t in w['terms']])
    out = []
    for records in (True, False):
        eng = _engine(max_width=max_width, records=records)
        terms = eng.edge_terms(G, w['gamma'], w['beta'])
        assert np.max(np.abs(terms - ref)) < TOL
        cfg = eng.compile(G, p, w['gamma'], w['beta']).plan.last_launch_config()
        assert any(c[3] & 128 for c in cfg) == records
        out.append(terms)
    assert np.max(np.abs(out[0] - out[1])) < 1e-6


@pytest.mark.parametrize('name,p,max_width', [('cfg3', 3, 29), ('cfg4', 4, 29), ('cfg2', 3, 11)])
def test_warp_queue_records_match_blob_path(cuda_device, monkeypatch, name, p, max_width):
    """The warp-per-network queue contracting from compact element records
    (each warp's own gate-table copy before its arena) gives the reference's
    edge terms and the terms of the same queue staging plan blobs (records
    off): N=1000 p=3 (every network has compact records, so the queue runs
    on them), N=256 p=4 (wide networks beside it in waves; its queue also
    holds networks with wide-format records, so it stages blobs either
    way), N=100 p=3 sliced below its width."""
    monkeypatch.setenv('QTB_SCHEDULE', 'warp:64')   # two warp slots fit a CTA on every workload
    G, w = golden_graph(name)
    ref = np.array([complex(*t) for t in w['terms']])
    out = []
    for records in (True, False):
        eng = _engine(max_width=max_width, records=records)
        terms = eng.edge_terms(G, w['gamma'], w['beta'])
        assert np.max(np.abs(terms - ref)) < TOL
        cg = eng.compile(G, p, w['gamma'], w['beta'])
        warp = [c for c in cg.plan.last_launch_config() if c[3] & 16]
        assert len(warp) == 1
        if not records or name == 'cfg3':
            assert bool(warp[0][3] & 128) == records
        E = eng.energy_expectation(G, w['gamma'], w['beta'])
        assert abs(E - w['energy']) <= TOL * abs(w['energy'])
        assert cg.plan.device_status() == 0
        out.append(terms)
    assert np.max(np.abs(out[0] - out[1])) < 1e-6


def test_reference_named_simulator(cuda_device):
    """QAOAQtreeSimulator under the reference's method names, returning the
    reference's result shape: a one-element float64 array for a graph with
    edges (qtensor/QAOASimulator.py:27-41,65), 0.0 without edges."""
    import networkx as nx
    from qtensor_b200.qaoa import QAOAQtreeSimulator
    G, w = golden_graph('cfg2')
    sim = QAOAQtreeSimulator('default')
    for E in (sim.energy_expectation(G, w['gamma'], w['beta']),
              sim.energy_expectation_parallel(G, w['gamma'], w['beta'], n_processes=8),
              sim.energy_expectation_mpi(G, w['gamma'], w['beta'])):
        assert isinstance(E, np.ndarray) and E.shape == (1,) and E.dtype == np.float64
        assert abs(E[0] - w['energy']) <= TOL * abs(w['energy'])
    empty = nx.empty_graph(5)
    assert sim.energy_expectation(empty, [0.1], [0.2]) == 0.0


def test_composers_agree_and_terms_are_real(cuda_device):
    """The reference's consistency checks: simplified (default), ZZ and CX
    circuits give the same energy (qtensor/tests/test_simplify_circuit.py,
    test_composers.py), and every edge term is real (test_simulators.py:68-85)."""
    G, w = golden_graph('cfg2')
    energies = []
    for comp in ('default', 'zz', 'cx'):
        eng = _engine(composer=comp)
        terms = eng.edge_terms(G, w['gamma'], w['beta'])
        assert np.max(np.abs(terms.imag)) < TOL
        energies.append(eng.energy_expectation(G, w['gamma'], w['beta']))
    assert max(energies) - min(energies) <= TOL * abs(w['energy'])


def test_edge_cases_follow_the_reference(cuda_device):
    """Edge cases with the reference's answers (oracle port): p = 0 (only the
    Hadamard layer: every <ZZ> is 0, energy |E|/2), a graph without edges
    (an empty sum: 0), isolated nodes and a single edge."""
    import networkx as nx
    import qtensor_port as port
    eng = _engine()
    G = graphs.regular(10, seed=1)
    assert abs(eng.energy_expectation(G, [], []) - G.number_of_edges() / 2) < TOL
    assert eng.energy_expectation(nx.empty_graph(5), [0.3], [0.2]) == 0.0
    assert len(eng.edge_terms(nx.empty_graph(5), [0.3], [0.2])) == 0
    H = nx.Graph([(0, 1)])
    H.add_nodes_from([2, 3])
    g, b = graphs.angles(2, seed=3)
    ref = float(np.real(np.ravel(port.energy_expectation(H, g, b))[0]))
    assert abs(eng.energy_expectation(H, g, b) - ref) <= TOL * max(1.0, abs(ref))
    with pytest.raises(ValueError):
        eng.energy_expectation(G, [0.1], [])


def test_scratch_bytes_same_before_and_after_upload(cuda_device):
    """The pre-upload size (used by the server's admission) is the size the
    uploaded plan's run needs."""
    from qtensor_b200.plan import NetworkPlan, graph_csr
    G, w = golden_graph('cfg4')
    params = np.concatenate([w['gamma'], w['beta']])
    plan = NetworkPlan(8)
    plan.add_lightcones(graph_csr(G), np.array(list(G.edges())), 4, 0, params)
    before = plan.scratch_bytes(0, len(plan))
    plan.upload()
    assert plan.scratch_bytes(0, len(plan)) == before > 0


def test_shared_lightcones_match_own_compiles_on_device(cuda_device):
    """On the device, a plan whose isomorphic lightcones share one compile
    (and one blob) gives every edge the term of a plan that compiles every
    edge from its own lightcone, and both match the reference fixture."""
    from qtensor_b200.plan import NetworkPlan, graph_csr
    G, w = golden_graph('cfg2')
    params = np.concatenate([w['gamma'], w['beta']])
    ref = np.array([complex(*t) for t in w['terms']])
    params_dev = torch.from_numpy(params).to(cuda_device)
    out = []
    for share in (True, False):
        plan = NetworkPlan(6)
        plan.set_order_trials(4)
        plan.set_share_lightcones(share)
        plan.add_lightcones(graph_csr(G), np.array(list(G.edges())), 3, 0, params)
        plan.upload()
        n = len(plan)
        terms = torch.empty(n, dtype=torch.complex64, device=cuda_device)
        nbytes = plan.scratch_bytes(0, n)
        scratch = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=cuda_device) if nbytes else None
        plan.run(0, n, params_dev, terms, None, scratch, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert plan.device_status() == 0
        out.append(terms.cpu().numpy())
        if share:
            ex = plan.export()
            assert len(set(ex['runs']['blob_off16'].tolist())) < n     # blobs are shared
    assert np.max(np.abs(out[0] - ref)) < 1e-5
    assert np.max(np.abs(out[1] - ref)) < 1e-5
    assert np.max(np.abs(out[0] - out[1])) < 2e-6
