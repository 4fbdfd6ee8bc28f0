"""Edge-sharded QAOA energies over ``torch.distributed`` ranks, one GPU each.

Edge terms are independent (qtensor/QAOASimulator.py:80-85, the edge fan-out
of ``energy_expectation_parallel`` and ``energy_expectation_mpi``
:72-108), so every rank contracts its own share of the edges on its own GPU
and the only exchange is one all-reduce of the ranks' fp64 energy shares
(8 bytes each).  ``energy_expectation_mpi`` hands the result to rank 0 only;
here every rank receives it.

Shares: ``shard_edges`` assigns edge i to rank ``i % world`` (random graphs
balance well that way); ``lpt_shards`` assigns by longest processing time
first when per-edge costs are known (e.g. the plans' algorithmic flops).
"""
import heapq

import numpy as np
import torch


def shard_edges(n_edges, rank, world):
    """Indices of the edges rank ``rank`` of ``world`` contracts (strided)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError('rank {} outside a world of {}'.format(rank, world))
    return list(range(rank, n_edges, world))


def lpt_shards(costs, world):
    """Longest-processing-time assignment: edges in descending cost, each to
    the rank with the least total so far.  Returns one index list per rank,
    each in ascending edge order."""
    heap = [(0.0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shards]


def sharded_energy(G, gamma, beta, partial_energy, group=None, shards=None, device=None,
                   n_edges=None):
    """Energy of ``G`` from the ranks' shares.

    partial_energy(G, gamma, beta, edges) -> float: this rank's share,
    ``(len(edges) - Re sum of their edge terms) / 2``; it is called with an
    empty list on a rank that has no edges.  shards: one edge-index list per
    rank (default ``shard_edges``).  device: where the all-reduce tensor
    lives (a CUDA device for NCCL; CPU for gloo).  n_edges: G's edge count
    when the caller knows it (networkx counts edges in O(nodes)).  Every
    rank takes part in the same single all-reduce, also when its share is
    empty."""
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    n = G.number_of_edges() if n_edges is None else n_edges
    mine = shard_edges(n, rank, world) if shards is None else shards[rank]
    share = float(partial_energy(G, gamma, beta, mine)) if mine else 0.0
    t = torch.tensor([share], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())


class DistributedQAOAEnergy:
    """``energy_expectation`` of ``QAOAEnergyEngine`` with the edges sharded
    over the ranks of ``group`` (NCCL, one GPU per rank).  Plans of a rank's
    share are compiled and cached on that rank only."""

    def __init__(self, group=None, lpt=False, **engine_kw):
        from .engine import QAOAEnergyEngine
        self.group = group
        self.lpt = lpt
        self.engine = QAOAEnergyEngine(**engine_kw)
        self._shards = {}

    def _shards_for(self, G, p, gamma, beta):
        """One tuple of edge indices per rank, kept per graph (the same
        tuple every call, so the engine hashes a share once): LPT from the
        plans' algorithmic flops (every rank compiles the whole graph once
        to cost it), or strided."""
        key = self.engine._key(G, p)
        if key not in self._shards:
            import torch.distributed as dist
            world = dist.get_world_size(self.group)
            if self.lpt:
                cg = self.engine.compile(G, p, gamma, beta)
                costs = np.zeros(cg.n_edges)
                for g, info in zip(cg.groups - cg.groups[0], cg.infos):
                    costs[g] += info['alg_flops']
                shards = lpt_shards(costs, world)
            else:
                n = self.engine._n_edges(G)
                shards = [shard_edges(n, r, world) for r in range(world)]
            if len(self._shards) >= 64:
                self._shards.pop(next(iter(self._shards)))
            self._shards[key] = [tuple(s) for s in shards]
        return self._shards[key]

    def energy_expectation(self, G, gamma, beta):
        p = len(np.asarray(gamma).ravel())
        shards = self._shards_for(G, p, gamma, beta)

        def share(G_, gamma_, beta_, edges):
            return self.engine.energy_expectation(G_, gamma_, beta_, edges=edges)

        return sharded_energy(G, gamma, beta, share, self.group, shards, device=self.engine.device,
                              n_edges=self.engine._n_edges(G))
