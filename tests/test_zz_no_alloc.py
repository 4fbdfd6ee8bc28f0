"""The allocation-free entry point ``qtb_plan_run_noalloc`` against the
regular ``qtb_plan_run``.

It serves callers that must not allocate device memory while they run (a
framework that owns all device allocations through its own pool, or a
process held to a fixed device-memory budget): it keeps arenas, job list
and completion counter in a static device array instead of allocating.
Kept in a file of its own that pytest collects last, and independent of the
other tests' state.
"""
import ctypes

import numpy as np
import pytest
import torch

import graphs
from conftest import golden_graph

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _compiled(G, p, params):
    from qtensor_b200 import _lib
    from qtensor_b200.plan import NetworkPlan, graph_csr
    _lib.check(_lib.lib().qtb_init(0))
    plan = NetworkPlan(2 * p)
    plan.set_order_trials(16)
    plan.add_lightcones(graph_csr(G), np.array(list(G.edges())), p, 0, params)
    plan.upload()
    return plan


def _run_regular(plan, n, params_dev, dev):
    terms = torch.empty(n, dtype=torch.complex64, device=dev)
    energy = torch.empty(1, dtype=torch.float64, device=dev)
    nbytes = plan.scratch_bytes(0, n)
    scratch = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=dev) if nbytes else None
    plan.run(0, n, params_dev, terms, energy, scratch, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return terms.cpu().numpy(), float(energy.item())


def _run_noalloc(plan, n, params_dev, dev):
    """One call through the C ABI into caller-owned outputs; returns the
    terms, the energy and the device's free bytes before and after the
    call (cudaMemGetInfo, synchronised on both sides)."""
    from qtensor_b200 import _lib
    terms = torch.empty(n, dtype=torch.complex64, device=dev)
    energy = torch.empty(1, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    _lib.check(_lib.lib().qtb_plan_run_noalloc(
        plan._h, 0, n, ctypes.c_void_p(params_dev.data_ptr()), ctypes.c_void_p(terms.data_ptr()),
        ctypes.c_void_p(energy.data_ptr()),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info(dev)[0]
    return terms.cpu().numpy(), float(energy.item()), (free_before, free_after)


def test_noalloc_matches_regular_run_twice(cuda_device):
    G, w = golden_graph('cfg2')
    p = 3
    plan = _compiled(G, p, np.concatenate([w['gamma'], w['beta']]))
    n = G.number_of_edges()
    ref_terms = np.array([complex(*t) for t in w['terms']])
    for k, seed in enumerate((11, 12)):     # two calls in a row, different angles
        params = np.concatenate(graphs.angles(p, seed=seed))
        params_dev = torch.from_numpy(params).to(cuda_device)
        t_reg, e_reg = _run_regular(plan, n, params_dev, cuda_device)
        t_na, e_na, (free0, free1) = _run_noalloc(plan, n, params_dev, cuda_device)
        assert np.max(np.abs(t_na - t_reg)) < TOL
        assert abs(e_na - e_reg) <= TOL * abs(e_reg)
        if k > 0:        # after the first call's set-up, device memory in use is unchanged
            assert free1 == free0
    assert plan.device_status() == 0
    # and the fixture's own angles reproduce the reference's edge terms
    params_dev = torch.from_numpy(np.concatenate([w['gamma'], w['beta']])).to(cuda_device)
    t_na, e_na, (free0, free1) = _run_noalloc(plan, n, params_dev, cuda_device)
    assert free1 == free0
    assert np.max(np.abs(t_na - ref_terms)) < TOL
    assert abs(e_na - w['energy']) <= TOL * abs(w['energy'])


def test_noalloc_rejects_requests_beyond_the_static_scratch(cuda_device):
    from qtensor_b200 import _lib
    G, w = golden_graph('cfg4')
    plan = _compiled(G, 4, np.concatenate([w['gamma'], w['beta']]))
    n = G.number_of_edges()
    terms = torch.empty(n, dtype=torch.complex64, device=cuda_device)
    params_dev = torch.zeros(8, dtype=torch.float64, device=cuda_device)
    code = _lib.lib().qtb_plan_run_noalloc(plan._h, 0, n, ctypes.c_void_p(params_dev.data_ptr()),
                                           ctypes.c_void_p(terms.data_ptr()), None, None)
    assert code == _lib.QTB_ERR_UNSUPPORTED
    assert 'split the range' in _lib.last_error()
