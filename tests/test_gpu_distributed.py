"""Edge shares on the GPU: disjoint shares add up to the energy, and the
sharded entry point over a one-rank NCCL group equals the engine's energy."""
import socket

import pytest

from conftest import golden_graph

pytestmark = pytest.mark.gpu


def test_edge_shares_add_up(cuda_device):
    from qtensor_b200.engine import QAOAEnergyEngine
    G, w = golden_graph('cfg2')
    eng = QAOAEnergyEngine()
    full = eng.energy_expectation(G, w['gamma'], w['beta'])
    n = G.number_of_edges()
    shares = [eng.energy_expectation(G, w['gamma'], w['beta'], edges=range(r, n, 3)) for r in range(3)]
    assert abs(sum(shares) - full) < 1e-9 * n
    assert abs(full - w['energy']) <= 1e-5 * abs(w['energy'])


@pytest.mark.parametrize('lpt', [False, True])
def test_distributed_energy_one_rank_nccl(cuda_device, lpt):
    import torch.distributed as dist
    from qtensor_b200.distributed import DistributedQAOAEnergy
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    dist.init_process_group('nccl', init_method='tcp://127.0.0.1:{}'.format(port), rank=0, world_size=1)
    try:
        G, w = golden_graph('cfg2')
        E = DistributedQAOAEnergy(lpt=lpt).energy_expectation(G, w['gamma'], w['beta'])
    finally:
        dist.destroy_process_group()
    assert abs(E - w['energy']) <= 1e-5 * abs(w['energy'])
