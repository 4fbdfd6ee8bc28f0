"""Edge sharding across ranks (host logic, CPU): shard maps and the one
all-reduce of fp64 energy shares, run as world-size-2 gloo process groups
with the oracle port contracting each rank's edges."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from qtensor_b200.distributed import lpt_shards, shard_edges


def test_strided_shards_partition_the_edges():
    for n in (0, 1, 7, 30):
        for world in (1, 2, 3, 8):
            shards = [shard_edges(n, r, world) for r in range(world)]
            flat = sorted(i for s in shards for i in s)
            assert flat == list(range(n))
            assert max(map(len, shards)) - min(map(len, shards)) <= 1
    with pytest.raises(ValueError):
        shard_edges(5, 2, 2)


def test_lpt_shards_balance_costs():
    rng = np.random.default_rng(0)
    costs = rng.pareto(1.5, size=200) + 1
    shards = lpt_shards(costs, 4)
    assert sorted(i for s in shards for i in s) == list(range(200))
    loads = [sum(costs[i] for i in s) for s in shards]
    # LPT: the largest load exceeds the mean by at most the largest single cost
    assert max(loads) - np.mean(loads) <= costs.max() + 1e-9


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, graph_name, use_lpt, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, 'tests'), os.path.join(root, 'oracle')]
    import torch.distributed as dist
    import qtensor_port as qport
    from conftest import golden_graph
    from qtensor_b200.distributed import lpt_shards, sharded_energy

    dist.init_process_group('gloo', init_method='tcp://127.0.0.1:{}'.format(port),
                            rank=rank, world_size=world)
    try:
        G, w = golden_graph(graph_name)
        edges = list(G.edges())

        def share(G_, gamma, beta, idx):
            total = sum(complex(np.ravel(qport.edge_energy(G_, gamma, beta, edges[i]))[0]) for i in idx)
            return (len(idx) - total.real) / 2

        shards = lpt_shards(np.arange(len(edges), dtype=float) % 5 + 1, world) if use_lpt else None
        out.put((rank, sharded_energy(G, w['gamma'], w['beta'], share, shards=shards)))
    except Exception as exc:     # noqa: BLE001 - reported to the parent
        out.put((rank, exc))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('use_lpt', [False, True])
def test_sharded_energy_gloo_world2(use_lpt):
    """Both ranks receive the energy the reference computes serially."""
    from conftest import golden_graph
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port_no = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port_no, 'cfg1_default', use_lpt, out))
             for r in range(2)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    _, w = golden_graph('cfg1_default')
    assert set(results) == {0, 1}
    for e in results.values():
        assert not isinstance(e, Exception), e
        assert abs(e - w['energy']) < 1e-10 * abs(w['energy'])


def test_rank_without_edges_still_joins_the_reduce():
    """A graph with fewer edges than ranks: the empty rank contributes 0."""
    ctx = mp.get_context('spawn')
    out = ctx.Queue()
    port_no = _free_port()
    procs = [ctx.Process(target=_rank_single_edge, args=(r, 2, port_no, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for e in results.values():
        assert not isinstance(e, Exception), e
    assert results[0] == results[1] == pytest.approx(0.25)


def _rank_single_edge(rank, world, port, out):
    import networkx as nx
    import torch.distributed as dist
    from qtensor_b200.distributed import sharded_energy
    dist.init_process_group('gloo', init_method='tcp://127.0.0.1:{}'.format(port),
                            rank=rank, world_size=world)
    try:
        G = nx.Graph([(0, 1)])
        calls = []

        def share(G_, gamma, beta, idx):
            calls.append(list(idx))
            return 0.25

        e = sharded_energy(G, [0.1], [0.2], share)
        out.put((rank, e if calls == ([[0]] if rank == 0 else []) else AssertionError(calls)))
    except Exception as exc:     # noqa: BLE001 - reported to the parent
        out.put((rank, exc))
    finally:
        dist.destroy_process_group()

