"""The C++ plan compiler and the C ABI, checked on the CPU (no GPU needed):
elimination orders against the reference fixtures, and the compiled device
plans executed by a numpy interpreter against the reference amplitudes."""
import ctypes
import re

import numpy as np
import pytest

import graphs
import plan_interp
import qtensor_port as port
from conftest import ROOT, golden_graph
from qtensor_b200 import _lib
from qtensor_b200.lightcone import composer_id, reference_lightcone, simplify_passes
from qtensor_b200.plan import NetworkPlan, graph_csr


def _params(w):
    return np.concatenate([w['gamma'], w['beta']])


def _ref_plan(G, w, comp='default'):
    p = len(w['gamma'])
    plan = NetworkPlan(2 * p)
    for edge in G.edges():
        nq, gates = reference_lightcone(G, edge, p, comp)
        plan.add_circuit(nq, gates, _params(w), simplify_passes(comp))
    return plan


def test_library_exports_every_header_symbol():
    with open(f'{ROOT}/include/qtb.h') as f:
        header = f.read()
    declared = set(re.findall(r'\b(qtb_[a-z0-9_]+)\s*\(', header))
    lib = _lib.lib()
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(_lib.EXPORTS)
    assert b'sm_100a' in lib.qtb_version()


@pytest.mark.parametrize('comp', ['default', 'cx', 'zz'])
def test_reference_order_matches_fixture(comp):
    """Same greedy elimination order and width as the reference, edge by edge."""
    G, w = golden_graph('cfg1_' + comp)
    plan = _ref_plan(G, w, comp)
    for k in range(len(w['terms'])):
        assert plan.peo(k) == w['peo'][k]
        assert plan.info(k)['treewidth'] == w['widths'][k]


@pytest.mark.parametrize('name', ['cfg1_default', 'cfg1_cx', 'cfg1_zz', 'test_random_n4_p4_d3',
                                  'test_grid2d_n3_p3_d0', 'test_line_n8_p4_d0', 'petersen_p9'])
def test_interpreted_plan_matches_reference(name):
    G, w = golden_graph(name)
    plan = _ref_plan(G, w, w['composer'])
    vals = plan_interp.run_plan(plan, _params(w))
    ref = np.array([complex(*t) for t in w['terms']])
    assert np.max(np.abs(vals - ref)) < 1e-12


@pytest.mark.parametrize('comp', ['default', 'cx'])
def test_native_order_plan_matches_reference(comp):
    """Native (C++ lightcone) ordering: different numbering, same amplitudes."""
    G, w = golden_graph('cfg1_default')
    p = len(w['gamma'])
    plan = NetworkPlan(2 * p)
    csr = graph_csr(G)
    plan.add_lightcones(csr, np.array(list(G.edges())), p, composer_id(comp), _params(w))
    vals = plan_interp.run_plan(plan, _params(w))
    ref = np.array([complex(*t) for t in w['terms']])
    assert np.max(np.abs(vals - ref)) < 1e-12


def test_native_plan_cfg2_sample():
    G, w = golden_graph('cfg2')
    edges = list(G.edges())[::10]
    plan = NetworkPlan(6)
    plan.add_lightcones(graph_csr(G), np.array(edges), 3, 0, _params(w), threads=4)
    vals = plan_interp.run_plan(plan, _params(w))
    ref = np.array([complex(*w['terms'][k]) for k in range(0, len(w['edges']), 10)])
    assert np.max(np.abs(vals - ref)) < 1e-12


def test_native_plan_cfg3_shape():
    """All 1500 edge networks of the N=1000 p=3 workload compile; their
    widths are the reference's (same cones, greedy order up to numbering)."""
    G, w = golden_graph('cfg3')
    plan = NetworkPlan(6)
    plan.add_lightcones(graph_csr(G), np.array(list(G.edges())), 3, 0, _params(w))
    infos = plan.infos()
    assert len(infos) == 1500
    assert max(i['treewidth'] for i in infos) <= max(w['widths']) + 2
    assert all(i['arena_elems'] * 8 <= 200 * 1024 for i in infos)
    assert all(i['angle_specific'] == 0 for i in infos)


@pytest.mark.parametrize('name', ['cfg1_default', 'cfg1_cx', 'test_random_n4_p4_d3', 'test_grid2d_n3_p3_d0',
                                  'test_line_n8_p4_d0'])
def test_element_records_match_reference(name):
    """Every network's element records (resolved operand offsets in the
    shared window) give the reference amplitude, reading only elements
    written before them.  Networks whose arena cannot be in shared memory
    have none."""
    G, w = golden_graph(name)
    plan = _ref_plan(G, w, w['composer'])
    ex = plan.export()
    has = ex['runs']['rec_words'] > 0
    arena_bytes = 8 * ex['runs']['arena_elems'].astype(np.int64)
    assert np.any(has)
    assert np.all(has[arena_bytes <= 200 * 1024]) and not np.any(has[arena_bytes > 224 * 1024])
    formats = set(ex['runs']['rec_format'][has].tolist())
    if name == 'test_grid2d_n3_p3_d0':        # windows above and below 4096 elements
        assert formats == {_lib.REC_WIDE, _lib.REC_COMPACT}
    vals = plan_interp.run_plan(plan, _params(w), records=True)
    ref = np.array([complex(*t) for t in w['terms']])
    assert np.max(np.abs(vals - ref)) < 1e-12


def test_element_records_sliced_and_native():
    """Records of native-order and sliced networks (N=100 p=3 sample,
    forced below its width) sum to the reference terms."""
    G, w = golden_graph('cfg2')
    edges = list(G.edges())[::10]
    plan = NetworkPlan(6)
    plan.set_max_width(11)
    plan.add_lightcones(graph_csr(G), np.array(edges), 3, 0, _params(w), threads=4)
    assert max(i['n_slices'] for i in plan.infos()) > 1
    vals = plan_interp.run_plan(plan, _params(w), records=True)
    ref = np.array([complex(*w['terms'][k]) for k in range(0, len(w['edges']), 10)])
    assert np.max(np.abs(vals - ref)) < 1e-12


def test_element_records_follow_shared_blobs():
    """Networks with one blob share one copy of its records; with records
    off the plan has none."""
    G, w = golden_graph('cfg3')
    edges = np.array(list(G.edges())[:300])
    plan = NetworkPlan(6)
    plan.add_lightcones(graph_csr(G), edges, 3, 0, _params(w))
    runs = plan.export()['runs']
    assert np.all(runs['rec_words'] > 0)
    by_blob = {}
    for r in runs:
        by_blob.setdefault(int(r['blob_off16']), set()).add((int(r['rec_off']), int(r['rec_words'])))
    assert all(len(v) == 1 for v in by_blob.values())
    assert len({int(r['rec_off']) for r in runs}) == len(by_blob) < len(runs)
    off = NetworkPlan(6)
    off.set_records(False)
    off.add_lightcones(graph_csr(G), edges, 3, 0, _params(w))
    ex = off.export()
    assert len(ex['recs']) == 0 and np.all(ex['runs']['rec_words'] == 0)


def test_simplifier_keeps_reference_hadamard_merge():
    """The reference simplifier turns H.H on one qubit into a single H
    (simplify_circuit.py:69-70 with gates.py hadamard); the plan does too."""
    gates = np.array([(_lib.GATE_H, 0, -1, -1, 0.0), (_lib.GATE_H, 0, -1, -1, 0.0)],
                     dtype=_lib.GATE_DTYPE)
    plan = NetworkPlan(0)
    plan.add_circuit(1, gates, np.zeros(0), simplify_passes=1)
    val = plan_interp.run_plan(plan, np.zeros(0))[0]
    assert abs(val - 1 / np.sqrt(2)) < 1e-15
    qops = __import__('qtree').operators
    amp = port.simulate_amplitude(port.simplify_qtree_circuit([qops.H(0), qops.H(0)]))
    assert abs(amp[0] - val) < 1e-15


def test_angle_dependent_cancellation_is_flagged():
    """Two X rotations whose angles cancel numerically but not structurally."""
    gates = np.array([(_lib.GATE_H, 0, -1, -1, 0.0), (_lib.GATE_XPHASE, 0, -1, 0, 2.0),
                      (_lib.GATE_XPHASE, 0, -1, 1, 2.0), (_lib.GATE_Z, 0, -1, -1, 0.0)],
                     dtype=_lib.GATE_DTYPE)
    plan = NetworkPlan(2)
    plan.add_circuit(1, gates, np.array([0.25, -0.25]), simplify_passes=1)
    assert plan.info(0)['angle_specific'] == 1
    assert plan.params_valid(np.array([0.1, -0.1]))
    assert not plan.params_valid(np.array([0.1, 0.2]))


def test_invalid_circuits_raise():
    plan = NetworkPlan(1)
    bad_kind = np.array([(99, 0, -1, -1, 0.0)], dtype=_lib.GATE_DTYPE)
    with pytest.raises(_lib.QtbError):
        plan.add_circuit(1, bad_kind, np.zeros(1))
    bad_qubit = np.array([(_lib.GATE_H, 3, -1, -1, 0.0)], dtype=_lib.GATE_DTYPE)
    with pytest.raises(_lib.QtbError):
        plan.add_circuit(2, bad_qubit, np.zeros(1))
    no_param = np.array([(_lib.GATE_XPHASE, 0, -1, 5, 2.0)], dtype=_lib.GATE_DTYPE)
    with pytest.raises(_lib.QtbError):
        plan.add_circuit(1, no_param, np.zeros(1))
    G = graphs.regular(10)
    with pytest.raises(_lib.QtbError):
        plan.add_lightcones(graph_csr(G), np.array([[0, 1]]), 2, 0, np.zeros(4))   # 2p != 1
    assert len(plan) == 0


def test_bucket_desc_validation_without_device():
    """Argument checks of qtb_bucket_c64 run before any CUDA call."""
    lib = _lib.lib()
    desc = _lib.BucketDesc()
    desc.n_inputs = 0
    ptrs = (ctypes.c_void_p * 1)()
    assert lib.qtb_bucket_c64(ctypes.byref(desc), ptrs, ctypes.c_void_p(8), None) == 1
    desc.n_inputs, desc.n_vars, desc.sum_first = 1, 2, 1
    desc.masks[0] = 0b100          # names a variable outside the union
    ptrs[0] = 16
    assert lib.qtb_bucket_c64(ctypes.byref(desc), ptrs, ctypes.c_void_p(8), None) == 1
    assert 'outside the union' in _lib.last_error()


@pytest.mark.parametrize('name,max_width', [('cfg1_default', 3), ('cfg2', 11), ('test_grid2d_n3_p3_d0', 8)])
def test_sliced_networks_sum_to_reference(name, max_width):
    """Slicing (FeynmanSimulator's parallel variables, greedy max-degree
    choice): every circuit becomes 2^k networks whose amplitudes sum to the
    reference's edge term; sliced widths stay below max_width."""
    G, w = golden_graph(name)
    p = len(w['gamma'])
    plan = NetworkPlan(2 * p)
    plan.set_max_width(max_width)
    plan.add_lightcones(graph_csr(G), np.array(list(G.edges())), p, 0, _params(w))
    infos = plan.infos()
    assert max(i['n_slices'] for i in infos) > 1            # slicing happened
    assert all(i['treewidth'] < max_width for i in infos)
    groups = plan.groups()
    assert np.all(np.diff(groups) >= 0) and groups[-1] == len(w['terms']) - 1
    vals = plan_interp.run_plan(plan, _params(w))
    ref = np.array([complex(*t) for t in w['terms']])
    assert np.max(np.abs(vals - ref)) < 1e-12


def test_p0_lightcones_match_reference():
    """p = 0: the cone is the edge alone under the Hadamard layer, every
    <ZZ> is 0 and the energy is |E| / 2, as the reference computes it."""
    G = graphs.regular(10, seed=1)
    plan = NetworkPlan(0)
    plan.add_lightcones(graph_csr(G), np.array(list(G.edges())), 0, 0, np.zeros(0))
    vals = plan_interp.run_plan(plan, np.zeros(0))
    ref = float(np.real(np.ravel(port.energy_expectation(G, [], []))[0]))
    assert abs((G.number_of_edges() - vals.real.sum()) / 2 - ref) < 1e-12


def test_scratch_bytes_before_upload():
    """The scratch a run needs (arenas of networks too large for shared
    memory) is known before upload, so a server can budget it; on the
    N=256 p=4 workload it is the wide networks' arenas, at most 1 GiB
    plus the largest one."""
    G, w = golden_graph('cfg4')
    plan = NetworkPlan(8)
    plan.set_order_trials(4)
    plan.add_lightcones(graph_csr(G), np.array(list(G.edges())), 4, 0, _params(w))
    nbytes = plan.scratch_bytes(0, len(plan))
    arenas = np.array([8 * i['arena_elems'] for i in plan.infos()])
    assert 0 < nbytes <= arenas[arenas > 200 * 1024].sum() + 64 * 8 * len(arenas)
    assert nbytes <= (1 << 30) + arenas.max() + 512


def test_images_follow_networks_added_after_an_export():
    """The flattened images are built once and reused; networks added after
    an export (or a scratch sizing) appear in the next one, and the result
    equals a plan that compiled every edge at once."""
    G = graphs.regular(30, seed=3)
    edges = np.array(list(G.edges()))
    params = np.concatenate(graphs.angles(2, seed=5))
    split = NetworkPlan(4)
    split.set_share_lightcones(False)     # classes would differ between the two calls
    split.add_lightcones(graph_csr(G), edges[:20], 2, 0, params)
    first = split.export()
    split.scratch_bytes(0, len(split))
    split.add_lightcones(graph_csr(G), edges[20:], 2, 0, params)
    whole = NetworkPlan(4)
    whole.set_share_lightcones(False)
    whole.add_lightcones(graph_csr(G), edges, 2, 0, params)
    a, b = split.export(), whole.export()
    assert len(a['nets']) == len(edges) > len(first['nets'])
    for key in ('nets', 'ops', 'ins', 'phases', 'runs', 'blobs', 'recs'):
        assert np.array_equal(a[key], b[key]), key
    assert np.max(np.abs(plan_interp.run_plan(split, params) - plan_interp.run_plan(whole, params))) == 0


def _network_blobs(plan):
    ex = plan.export()
    runs, blobs = ex['runs'], ex['blobs']
    return [bytes(blobs[16 * int(r['blob_off16']):16 * int(r['blob_off16']) + int(r['blob_bytes'])])
            for r in runs]


def test_isomorphic_lightcones_share_one_compile():
    """On a ring every edge's lightcone is the same path, so with sharing
    every edge gets the first edge's networks (byte-identical blobs), and
    the edge terms equal the reference's with and without sharing."""
    import networkx as nx
    G = nx.cycle_graph(12)
    edges = np.array(list(G.edges()))
    gamma, beta = graphs.angles(2, seed=9)
    params = np.concatenate([gamma, beta])
    ref = np.array([complex(np.ravel(port.edge_energy(G, gamma, beta, tuple(e)))[0]) for e in edges])
    shared, own = NetworkPlan(4), NetworkPlan(4)
    own.set_share_lightcones(False)
    for plan in (shared, own):
        plan.add_lightcones(graph_csr(G), edges, 2, 0, params)
        assert np.max(np.abs(plan_interp.run_plan(plan, params) - ref)) < 1e-10
    assert len(set(_network_blobs(shared))) == 1
    assert len(set(_network_blobs(own))) > 1      # the wrap-around edge numbers its cone apart


@pytest.mark.parametrize('seed', [0, 1, 2])
def test_lightcone_sharing_keeps_every_edge_term(seed):
    """Random 3-regular and Erdos-Renyi graphs (cones with and without
    cycles): sharing changes no edge term, and on the 3-regular graph it
    finds isomorphic cones to share."""
    import networkx as nx
    for G in (graphs.regular(60, seed=seed), nx.erdos_renyi_graph(40, 3 / 39, seed=seed)):
        if G.number_of_edges() == 0:
            continue
        edges = np.array(list(G.edges()))
        params = np.concatenate(graphs.angles(2, seed=seed))
        vals = []
        for share in (True, False):
            plan = NetworkPlan(4)
            plan.set_share_lightcones(share)
            plan.add_lightcones(graph_csr(G), edges, 2, 0, params)
            vals.append(plan_interp.run_plan(plan, params))
        assert np.max(np.abs(vals[0] - vals[1])) < 1e-10
    plan = NetworkPlan(4)
    plan.add_lightcones(graph_csr(graphs.regular(60, seed=seed)),
                        np.array(list(graphs.regular(60, seed=seed).edges())), 2, 0, params)
    blobs = _network_blobs(plan)
    assert len(set(blobs)) < len(blobs)


def _share_partition(plan):
    """Edges grouped by the blob their networks point at (one network per edge)."""
    offs = plan.export()['runs']['blob_off16'].tolist()
    first = {}
    return [first.setdefault(o, i) for i, o in enumerate(offs)]


@pytest.mark.parametrize('seed', [3, 4])
def test_lightcone_classes_do_not_depend_on_node_labels(seed):
    """On trees the canonical key is label-free: relabelling the graph's
    nodes at random (edges kept in the same order) gives the same classes
    of shared edges, and the same edge terms."""
    import networkx as nx
    rng = np.random.default_rng(seed)
    T = nx.random_labeled_tree(60, seed=seed) if hasattr(nx, 'random_labeled_tree') \
        else nx.random_tree(60, seed=seed)
    perm = rng.permutation(60)
    T2 = nx.Graph()
    T2.add_nodes_from(sorted(int(perm[v]) for v in T.nodes()))
    edges = list(T.edges())
    T2.add_edges_from((int(perm[a]), int(perm[b])) for a, b in edges)
    params = np.concatenate(graphs.angles(2, seed=seed))
    plans = []
    for G, E in ((T, edges), (T2, [(int(perm[a]), int(perm[b])) for a, b in edges])):
        csr = graph_csr(G)
        index = {v: i for i, v in enumerate(csr[0])}
        plan = NetworkPlan(4)
        plan.add_lightcones(csr, np.array([(index[a], index[b]) for a, b in E], dtype=np.int32), 2, 0, params)
        plans.append(plan)
    assert _share_partition(plans[0]) == _share_partition(plans[1])
    assert len(set(_share_partition(plans[0]))) < len(edges)
    vals = [plan_interp.run_plan(pl, params) for pl in plans]
    assert np.max(np.abs(vals[0] - vals[1])) < 1e-10


@pytest.mark.parametrize('bad', [(3, 3), (3, 99), (-1, 2)])
def test_invalid_edge_fails_the_call_with_sharing(bad):
    """An invalid edge among valid ones fails the whole call, names the edge,
    and adds no network, with lightcone sharing on (the default)."""
    G = graphs.regular(10, seed=1)
    edges = np.array(list(G.edges()) + [bad], dtype=np.int32)
    plan = NetworkPlan(2)
    with pytest.raises(_lib.QtbError, match='edge {}: lightcone'.format(len(edges) - 1)):
        plan.add_lightcones(graph_csr(G), edges, 1, 0, np.zeros(2))
    assert len(plan) == 0


def _edge_plan(G, edge, p, max_width, max_slices, trials=8):
    csr = graph_csr(G)
    idx = {v: i for i, v in enumerate(csr[0])}
    plan = NetworkPlan(2 * p)
    plan.set_order_trials(trials)
    plan.set_max_width(max_width, max_slices)
    g, b = graphs.angles(p, seed=1)
    plan.add_lightcones(csr, np.array([[idx[edge[0]], idx[edge[1]]]], dtype=np.int32), p,
                        composer_id('default'), np.concatenate([g, b]), 1)
    return plan


def _widest_edge(G, p):
    """An edge of G whose lightcone the reference's greedy order makes
    widest (port of OrderingOptimizer, qtensor/optimisation/Optimizer.py:65-87)."""
    g, b = graphs.angles(p, seed=1)
    best = None
    for e in list(G.edges())[:12]:
        circ = port.lightcone_circuit(G, e, g, b)
        buckets, _, bra, ket = port.circuit_to_network(circ)
        _, width = port.order_network(buckets, bra, ket)
        if best is None or width > best[1]:
            best = (e, width)
    return best


def test_network_beyond_arena_limit_is_rejected_not_crashed():
    """A lightcone whose contraction needs an arena beyond 2^31 complex64
    elements fails to compile with QTB_ERR_UNSUPPORTED (it used to write
    arena offsets into the gate-table flag bit and crash the compiler).  The
    reference's own greedy order gives that edge a width of 40 or more: its
    NumpyBackend would have to allocate a 2^40-element tensor, so no exact
    bucket elimination answers it."""
    G = graphs.erdos_renyi(graphs.ER_P4_N109['n'], graphs.ER_P4_N109['seed'])
    edge, ref_width = _widest_edge(G, 4)
    assert ref_width >= 40
    with pytest.raises(_lib.QtbError) as exc:
        _edge_plan(G, edge, 4, max_width=0, max_slices=256)
    assert exc.value.code == _lib.QTB_ERR_UNSUPPORTED
    assert 'arena' in str(exc.value) or 'exceeds the limit' in str(exc.value)
    # with slicing the request fails fast, naming the width it would need
    with pytest.raises(_lib.QtbError) as exc:
        _edge_plan(G, edge, 4, max_width=29, max_slices=1024)
    assert exc.value.code == _lib.QTB_ERR_UNSUPPORTED and 'width' in str(exc.value)


def test_minfill_candidates_never_worse_than_greedy():
    """The native order search keeps the cheapest (sum of 2^width over
    eliminations) of the reference greedy order, randomized greedy orders
    and minimum-fill orders: edge by edge its width is at most the
    reference order's, and over the edges it moves fewer bytes."""
    G = graphs.erdos_renyi(graphs.ER_P3_N213['n'], graphs.ER_P3_N213['seed'])
    ref_bytes = nat_bytes = 0.0
    for e in list(G.edges())[:20]:
        try:
            ref = _edge_plan(G, e, 3, 0, 1, trials=0).info(0)
        except _lib.QtbError:
            continue     # the reference order is too wide to compile at all
        nat = _edge_plan(G, e, 3, 0, 1, trials=8).info(0)
        assert nat['treewidth'] <= ref['treewidth']
        ref_bytes += ref['alg_bytes']
        nat_bytes += nat['alg_bytes']
    assert nat_bytes < ref_bytes
