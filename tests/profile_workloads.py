"""Workloads for the ncu captures summarised under profiles/ (measurement
infrastructure, not collected as tests).  Each mode runs a small, fixed
amount of work and checks its result, so that the same command can run once
without the profiler and then under it.

    python tests/profile_workloads.py cfg3        # 3-regular N=1000 p=3, 20 executor steps
    python tests/profile_workloads.py er400       # Erdos-Renyi N=400 p=3 (wide networks), 3 runs
    python tests/profile_workloads.py cfg4        # 3-regular N=256 p=4, 5 executor steps
    python tests/profile_workloads.py bucket24    # one 24-variable bucket through qtb_bucket_c64, 5 runs
    python tests/profile_workloads.py plain_cfg1  # 3-regular N=20 p=1 through the plain per-bucket path
    python tests/profile_workloads.py aux         # allocation-free run (N=100 p=3) and the wait self-test
    python tests/profile_workloads.py contract    # tcontract contract-sum on the tensor cores, K=1024 F=2 M=N=1024

QTB_SCHEDULE (see qtb.cu) fixes the executor schedule, so that the
profiler's serialised replays cannot steer the autotuner.
"""
import ctypes
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, 'tests')]

import networkx as nx  # noqa: E402
import numpy as np  # noqa: E402
import torch  # noqa: E402

import graphs  # noqa: E402
from conftest import golden_graph  # noqa: E402
from qtensor_b200 import _lib  # noqa: E402
from qtensor_b200.engine import QAOAEnergyEngine  # noqa: E402


def cfg3():
    G, w = golden_graph('cfg3')
    eng = QAOAEnergyEngine()
    cg = eng.compile(G, 3, w['gamma'], w['beta'])
    cg.params.copy_(torch.from_numpy(np.concatenate([w['gamma'], w['beta']])))
    graph = cg.device_graph()
    for _ in range(20):
        graph.replay()
    torch.cuda.synchronize()
    E = float(cg.energy.cpu()[0])
    assert abs(E - w['energy']) <= 1e-5 * abs(w['energy']), (E, w['energy'])
    assert cg.plan.device_status() == 0
    print('launch classes', cg.plan.last_launch_config())


def cfg4():
    G, w = golden_graph('cfg4')
    eng = QAOAEnergyEngine()
    cg = eng.compile(G, 4, w['gamma'], w['beta'])
    cg.params.copy_(torch.from_numpy(np.concatenate([w['gamma'], w['beta']])))
    graph = cg.device_graph()
    for _ in range(5):
        graph.replay()
    torch.cuda.synchronize()
    E = float(cg.energy.cpu()[0])
    assert abs(E - w['energy']) <= 1e-5 * abs(w['energy']), (E, w['energy'])
    assert cg.plan.device_status() == 0
    print('launch classes', cg.plan.last_launch_config())


def er400():
    G = nx.erdos_renyi_graph(400, 3 / 399, seed=24323709)
    g, b = graphs.angles(3, seed=1)
    eng = QAOAEnergyEngine(autotune=False)
    cg = eng.compile(G, 3, g, b)
    cg.params.copy_(torch.from_numpy(np.concatenate([g, b])))
    for _ in range(3):
        cg.launch()
    torch.cuda.synchronize()
    assert cg.plan.device_status() == 0
    print('launch classes', cg.plan.last_launch_config())


def bucket24():
    """One bucket of 24 binary variables, variable 0 summed: A over every
    variable but the lowest (2^23 elements), B over variable 0 and the 12
    lowest (2^13), a gate over variable 0 and the lowest (2^2); output 2^23
    (64 MB read, 64 MB written)."""
    lib = _lib.lib()
    _lib.check(lib.qtb_init(0))
    u = 24
    masks = [((1 << u) - 1) & ~1, (1 << (u - 1)) | 0xfff, (1 << (u - 1)) | 1]
    gen = torch.Generator(device='cuda').manual_seed(0)
    ins = [torch.randn(1 << bin(m).count('1'), dtype=torch.complex64, device='cuda', generator=gen)
           for m in masks]
    out = torch.empty(1 << (u - 1), dtype=torch.complex64, device='cuda')
    desc = _lib.BucketDesc()
    desc.n_inputs, desc.n_vars, desc.sum_first = 3, u, 1
    for i, m in enumerate(masks):
        desc.masks[i] = m
    ptrs = (ctypes.c_void_p * 3)(*[x.data_ptr() for x in ins])
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(5):
        s.record()
        _lib.check(lib.qtb_bucket_c64(ctypes.byref(desc), ptrs, ctypes.c_void_p(out.data_ptr()),
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        e.record()
        e.synchronize()
        print('bucket %.1f us' % (1e3 * s.elapsed_time(e)))
    A, B, C = [x.cpu().numpy() for x in ins]
    o = out.cpu().numpy()

    def pext(x, m):
        r, bit = 0, 0
        for b in range(32):
            if (m >> b) & 1:
                r |= ((x >> b) & 1) << bit
                bit += 1
        return r
    for j in [0, 1, 12345, (1 << 23) - 1]:
        acc = 0
        for sbit in range(2):
            idx = j | (sbit << (u - 1))
            acc += A[pext(idx, masks[0])] * B[pext(idx, masks[1])] * C[pext(idx, masks[2])]
        assert abs(acc - o[j]) < 1e-3 * max(1, abs(acc)), (j, acc, o[j])


def plain_cfg1():
    G, w = golden_graph('cfg1_default')
    eng = QAOAEnergyEngine()
    for _ in range(2):
        t = eng.edge_terms(G, w['gamma'], w['beta'], path='plain')
        eng.energy_expectation(G, w['gamma'], w['beta'], path='plain')
    ref = np.array([complex(*x) for x in w['terms']])
    assert np.max(np.abs(t - ref)) < 1e-5


def aux():
    """qtb_plan_run_noalloc twice on the N=100 p=3 workload (its job kernel
    and executor) and the bounded-wait self-test kernel."""
    from qtensor_b200.plan import NetworkPlan, graph_csr
    lib = _lib.lib()
    _lib.check(lib.qtb_init(0))
    G, w = golden_graph('cfg2')
    params = np.concatenate([w['gamma'], w['beta']])
    plan = NetworkPlan(6)
    plan.add_lightcones(graph_csr(G), np.array(list(G.edges())), 3, 0, params)
    plan.upload()
    n = len(plan)
    dev = torch.device('cuda', 0)
    params_dev = torch.from_numpy(params).to(dev)
    terms = torch.empty(n, dtype=torch.complex64, device=dev)
    energy = torch.empty(1, dtype=torch.float64, device=dev)
    for _ in range(2):
        _lib.check(lib.qtb_plan_run_noalloc(
            plan._h, 0, n, ctypes.c_void_p(params_dev.data_ptr()), ctypes.c_void_p(terms.data_ptr()),
            ctypes.c_void_p(energy.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        torch.cuda.synchronize()
        assert abs(float(energy.item()) - w['energy']) <= 1e-5 * abs(w['energy'])
    status = ctypes.c_int32(0)
    _lib.check(lib.qtb_selftest_wait_timeout(1 << 12, ctypes.byref(status)))
    assert status.value == _lib.STATUS_WAIT_TIMEOUT


def contract():
    """C[f,m,n] = sum_k A[k,f,m] B[k,f,n] with K=1024, F=2, M=N=1024 (3xTF32
    on the tensor cores), 3 runs; checked against the CUDA-core path."""
    from qtensor_b200 import tcontract
    dev = torch.device('cuda', 0)
    K, F, M, N = 1024, 2, 1024, 1024
    gen = torch.Generator(device=dev).manual_seed(0)
    a = torch.randn((K, F, M), dtype=torch.complex64, device=dev, generator=gen)
    b = torch.randn((K, F, N), dtype=torch.complex64, device=dev, generator=gen)
    c = torch.empty((F, M, N), dtype=torch.complex64, device=dev)
    scratch = torch.empty(tcontract.contract_sum_scratch_bytes(K, F, M, N, 'tensor'), dtype=torch.uint8, device=dev)
    s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        s_.record()
        tcontract.mkl_contract_sum(a, b, c, mode='tensor', scratch=scratch)
        e_.record()
        e_.synchronize()
        ms = s_.elapsed_time(e_)
        print('contract-sum %.3f ms, %.1f TFLOP/s (8 M N K F useful flops)' % (ms, 8.0 * M * N * K * F / ms / 1e9))
    assert int(scratch[:4].view(torch.int32).item()) == 0
    ref = torch.empty_like(c)
    tcontract.mkl_contract_sum(a, b, ref, mode='simt')
    torch.cuda.synchronize()
    assert ((c - ref).abs().max() <= 1e-5 * ref.abs().max()).item()


if __name__ == '__main__':
    {'cfg3': cfg3, 'cfg4': cfg4, 'er400': er400, 'bucket24': bucket24, 'plain_cfg1': plain_cfg1,
     'aux': aux, 'contract': contract}[sys.argv[1]]()
    print('ok', sys.argv[1])
