"""QAOA edge-term throughput on B200 -- one JSON line on rank 0.

Workload (default): QAOA MaxCut energy, random 3-regular graph N=1000
(networkx seed 0 + rank), p=3, angles U[0, pi) drawn per step, default
composer (ZZ gates + commutation simplifier), greedy elimination order --
1500 edge-term networks per step.  One step = one full energy: gate tensors
generated from the step's 6 angles, all 1500 lightcone networks contracted,
fp64 compensated reduction to the energy.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

* ``value``: device-resident throughput (plans and angles already in HBM),
  CUDA events around each step on the launching stream, L2 flushed between
  steps (256 MiB write, outside the events); max over ranks.
* ``e2e``: the public API ``QAOAEnergyEngine.energy_expectation(G, gamma,
  beta)`` per step with host angles: pinned H2D of the angles and D2H of the
  energy inside the events; plans cached from the warm-up (a new graph's plan
  compile is reported separately as ``compile_s``).
* ``--impl reference``: the reference algorithm (the oracle port of QTensor's
  ``energy_expectation_parallel`` with its NumpyBackend, complex128 einsum)
  on all host cores, rank 0 only.
Multi-GPU (torchrun): every rank contracts its own graph (weak scaling); no
collective on the data path.  ``--shard`` instead shards one Erdos-Renyi
graph's edges over the ranks with one NCCL all-reduce per energy (strong
scaling, its own JSON line).

Extra legs on one GPU (rank 0): the reference greedy order, 3-regular N=256
p=4 with its error against the complex128 fixture, the recorded reference
driver's backend calls replayed into the drop-in backend, the plain
per-bucket path, the serving stream, and (``--serving-saturate N``) the
serving workload offered above the server's capacity.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, 'tests'))

import numpy as np  # noqa: E402

import graphs  # noqa: E402

METRIC = 'QAOA edge terms/s (3-regular N=1000 p=3)'
UNIT = 'edge terms/s'
PUBLISHED_TERMS_PER_S = 1500 / 4.89   # the reference's published N=1000 p=3 energy: 4.89 s on 56 processes
WORKLOAD = {'workload': 'qaoa-maxcut energy, random 3-regular N=1000 (seed 0+rank), p=3, '
                        'default composer, greedy order; 1500 edge-term networks per step',
            'graph_nodes': 1000, 'p': 3, 'edges': 1500, 'composer': 'default',
            'ordering': 'native'}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3000)
    ap.add_argument('--warmup', type=int, default=20)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--nodes', type=int, default=1000)
    ap.add_argument('--p', type=int, default=3)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--plain-steps', type=int, default=3,
                    help='steps of the plain per-bucket comparison (0 skips it)')
    ap.add_argument('--serving-requests', type=int, default=128,
                    help='requests of the serving run (0 skips it)')
    ap.add_argument('--serving-rate', type=float, default=20.0,
                    help='Poisson arrival rate of the serving run, requests/s')
    ap.add_argument('--serving-saturate', type=int, default=0,
                    help='requests of an extra serving run offered faster than the server '
                         'completes them (0 skips it; the stated stream is 10000)')
    ap.add_argument('--serving-saturate-rate', type=float, default=2000.0,
                    help='arrival rate of the saturation run, requests/s')
    ap.add_argument('--cfg4-steps', type=int, default=10,
                    help='steps of the 3-regular N=256 p=4 leg (0 skips it)')
    ap.add_argument('--reference-order-steps', type=int, default=10,
                    help='steps of the leg with the reference greedy order (0 skips it)')
    ap.add_argument('--no-tensor-core', action='store_true',
                    help='skip the tensor-core contract-sum leg')
    ap.add_argument('--no-dropin', action='store_true',
                    help="skip the replay of the reference driver's recorded backend calls")
    ap.add_argument('--shard', action='store_true',
                    help='under torchrun: shard one graph\'s edges over the ranks (one NCCL '
                         'all-reduce per energy) instead of one graph per rank')
    ap.add_argument('--shard-nodes', type=int, default=400,
                    help='Erdos-Renyi graph size of the sharded mode (p=3)')
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get('RANK', 0))
    world = int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))
    return rank, world, local


# ------------------------------------------------------------------ CPU arm
def cpu_reference(G, p, n_edges, seed, start_method):
    """Time the oracle port of the reference path on the host cores over the
    first ``n_edges`` edges.  Returns (terms/s, cores, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import qtensor_port as port
    cores = os.cpu_count() or 1
    gamma, beta = graphs.angles(p, seed)
    edges = list(G.edges())[:n_edges]
    t0 = time.perf_counter()
    port.energy_expectation_parallel(G, gamma, beta, n_processes=cores, edges=edges,
                                     start_method=start_method)
    dt = time.perf_counter() - t0
    return len(edges) / dt, cores, dt


def cpu_single_process(G, p, n_edges, seed):
    """The oracle port's serial edge loop (one process) over the first
    ``n_edges`` edges.  Returns (terms/s, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import qtensor_port as port
    gamma, beta = graphs.angles(p, seed)
    edges = list(G.edges())[:n_edges]
    t0 = time.perf_counter()
    for e in edges:
        port.edge_energy(G, gamma, beta, e)
    dt = time.perf_counter() - t0
    return len(edges) / dt, dt


def cpu_sample_edges(total):
    cores = os.cpu_count() or 1
    # about 0.03 s of single-core work per N=1000 p=3 edge: aim at ~15 s of work
    return int(min(total, max(64, 500 * cores)))


def run_reference(args, budget_s=150.0):
    """The reference arm: the oracle port of energy_expectation_parallel
    (NumpyBackend einsum, complex128) on every host core, rank 0 only.  One
    fork pool serves all steps; each step contracts a bounded sample of the
    workload's edges (rotating through all of them), sized from a
    calibration step so that warm-up and timed steps together take about
    `budget_s` seconds whatever --steps is; at least two edges per process."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from multiprocessing import get_context
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import qtensor_port as port
    G = graphs.regular(args.nodes, seed=0)
    edges = list(G.edges())
    cores = os.cpu_count() or 1
    with get_context('fork').Pool(cores) as pool:
        cursor = 0

        def step(n, seed):
            nonlocal cursor
            gamma, beta = graphs.angles(args.p, seed)
            sample = [edges[(cursor + i) % len(edges)] for i in range(n)]
            cursor = (cursor + n) % len(edges)
            tasks = [(G, gamma, beta, e, 'default') for e in sample]
            t0 = time.perf_counter()
            pool.map(port._edge_task, tasks, chunksize=max(1, n // (4 * cores)))
            return time.perf_counter() - t0

        rate = cores / step(cores, 0)                   # calibration, untimed
        per_step = budget_s / max(1, args.warmup + args.steps)
        # at least two edges per process, so that every core stays busy
        n_edges = int(min(len(edges), max(2 * cores, round(rate * per_step))))
        total_t, total_n = 0.0, 0
        for i in range(args.warmup + args.steps):
            dt = step(n_edges, i + 1)
            if i >= args.warmup:
                total_t += dt
                total_n += n_edges
    mean = total_t / max(1, args.steps)
    value = total_n / total_t
    sample = '{} of {} edges per step (rotating through all), oracle port of ' \
             'energy_expectation_parallel (NumpyBackend einsum, complex128), one fork pool of ' \
             '{} processes'.format(n_edges, len(edges), cores)
    line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': mean * 1e3,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': value / PUBLISHED_TERMS_PER_S,
            'dtype': 'c128', 'data': 'synthetic', 'impl': 'reference',
            'config': dict(WORKLOAD, ordering='reference greedy', cpu_sample=sample),
            'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': cores, 'kind': 'port',
                             'sample': sample},
            'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + self.FIELDS,
                 '--format=csv,noheader,nounits', '-lms', '200'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sms, maxes, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in self.lines:
            parts = [x.strip() for x in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxes.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == 'active':
                    reasons.add(name)
        return {'sm_mhz': statistics.median(sms) if sms else None,
                'sm_max_mhz': max(maxes) if maxes else None,
                'reasons': sorted(reasons), 'samples': len(sms)}


# ------------------------------------------------------------------ serving
def serving_requests(n, seed=0):
    """The serving workload: 3-regular or Erdos-Renyi (mean degree 3)
    graphs, N uniform in 16..500, p uniform in 1..4, angles U[0, pi)."""
    import networkx as nx
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        N = int(rng.integers(16, 501))
        p = int(rng.integers(1, 5))
        if rng.random() < 0.5:
            G = nx.random_regular_graph(3, N + (N % 2), seed=int(rng.integers(1 << 30)))
        else:
            G = nx.erdos_renyi_graph(N, 3 / (N - 1), seed=int(rng.integers(1 << 30)))
        if G.number_of_edges():
            gamma, beta = graphs.angles(p, seed=int(rng.integers(1 << 30)))
            out.append((G, gamma, beta))
    return out


# Contraction work a serving request may bring (algorithmic bytes): about
# two seconds of the wide-network executor; the one request of the 128-request
# stream above it (Erdos-Renyi N=73 p=4, 72 TB) would hold the GPU for a minute.
SERVING_MAX_REQUEST_BYTES = 4e12


def _pct(values, q):
    return float(np.percentile(values, q)) if len(values) else None


def _rejections(results):
    """Failed requests by cause: lightcones too wide for any exact
    contraction within the slice budget, over the work budget, other."""
    from qtensor_b200._lib import QtbError
    from qtensor_b200.serve import RequestTooLarge
    out = {'too_wide': 0, 'over_work_budget': 0, 'other': 0}
    for r in results:
        if isinstance(r, RequestTooLarge):
            out['over_work_budget'] += 1
        elif isinstance(r, QtbError) and 'width' in str(r):
            out['too_wide'] += 1
        elif isinstance(r, Exception):
            out['other'] += 1
    return out


def _available_cpus():
    from qtensor_b200._lib import available_cpus
    return available_cpus()


def summarize_serving(results, wall):
    ok = [r for r in results if not isinstance(r, Exception)]
    lat = np.array([r.latency for r in ok]) * 1e3
    edges = sum(r.edges for r in ok)
    out = {'completed': len(ok), 'rejected': len(results) - len(ok),
           'rejected_by_cause': _rejections(results),
           'p50_ms': _pct(lat, 50), 'p95_ms': _pct(lat, 95), 'p99_ms': _pct(lat, 99),
           'edge_terms_per_s': edges / wall if wall > 0 else None, 'wall_s': wall}
    # where the median request's time went
    for name in ('compile_s', 'wait_s', 'gpu_s'):
        vals = np.array([getattr(r, name) for r in ok]) * 1e3
        out['p50_' + name[:-2] + '_ms'] = _pct(vals, 50)
        out['max_' + name[:-2] + '_ms'] = float(vals.max()) if len(vals) else None
    return out


def run_serving_saturated(n_requests, rate, device_index):
    """The serving workload offered faster than the server completes it
    (Poisson arrivals at ``rate``, far above its capacity): the edge terms/s
    are then the server's sustained throughput, not the arrival rate."""
    from qtensor_b200.serve import QAOAServer
    reqs = serving_requests(n_requests, seed=2)
    gaps = np.random.default_rng(3).exponential(1.0 / rate, size=len(reqs))
    with QAOAServer(device=device_index, n_streams=8, compile_workers=4,
                    max_request_bytes=SERVING_MAX_REQUEST_BYTES) as srv:
        t0 = time.perf_counter()
        futs = []
        for r, gap in zip(reqs, gaps):
            time.sleep(gap)
            futs.append(srv.submit(*r))
        out = []
        for f in futs:
            try:
                out.append(f.result(timeout=3600))
            except Exception as exc:     # noqa: BLE001 - rejected (too wide, over budget)
                out.append(exc)
        wall = time.perf_counter() - t0
    res = summarize_serving(out, wall)
    res['workload'] = ('{} requests of the serving distribution (seed 2), Poisson arrivals at {} req/s '
                       '(seed 3); 8 streams, 4 compile workers').format(len(reqs), rate)
    return res


def run_serving(n_requests, rate, device_index, plain_budget_s=20.0):
    """Poisson stream through the continuous-batching server; the same
    stream through a FIFO queue (one compile worker, one stream); the same
    requests one at a time on a single-stream server; and, as the drop-in
    comparison, requests one at a time through the plain backend (one
    bucket-kernel launch per bucket, compile included) until about
    ``plain_budget_s`` seconds have passed."""
    from qtensor_b200.engine import QAOAEnergyEngine
    from qtensor_b200.serve import QAOAServer
    reqs = serving_requests(n_requests)
    rng = np.random.default_rng(1)
    gaps = rng.exponential(1.0 / rate, size=len(reqs))
    pct = _pct
    summarize = summarize_serving
    budget = SERVING_MAX_REQUEST_BYTES

    def collect(futs):
        out = []
        for f in futs:
            try:
                out.append(f.result(timeout=600))
            except Exception as exc:     # noqa: BLE001 - rejected (too wide, over budget)
                out.append(exc)
        return out

    warm_reqs = serving_requests(6, seed=7)

    def warm(srv):
        """Untimed, before a server's timed requests: a few requests of the
        same distribution (another seed), so that one-time costs (kernel
        modules loaded on first launch, allocator pools, worker start-up)
        fall outside every policy's numbers alike."""
        collect([srv.submit(*r) for r in warm_reqs])

    def poisson(srv):
        warm(srv)
        t0 = time.perf_counter()
        futs = []
        for (G, gamma, beta), gap in zip(reqs, gaps):
            time.sleep(gap)
            futs.append(srv.submit(G, gamma, beta))
        out = collect(futs)
        return out, time.perf_counter() - t0

    with QAOAServer(device=device_index, n_streams=4, max_request_bytes=budget) as srv:
        stream, wall_stream = poisson(srv)
    # the same arrivals through a plain FIFO queue: one compile worker, one
    # request on the GPU at a time
    # one request at a time on the GPU: its wide waves may take whole SMs
    with QAOAServer(device=device_index, n_streams=1, compile_workers=1, max_request_bytes=budget,
                    wave_ctas_per_sm=0) as srv:
        fifo, wall_fifo = poisson(srv)
    with QAOAServer(device=device_index, n_streams=1, compile_workers=1, max_request_bytes=budget,
                    wave_ctas_per_sm=0) as srv:
        warm(srv)
        t0 = time.perf_counter()
        alone = []
        for r in reqs:
            alone.extend(collect([srv.submit(*r)]))
        wall_alone = time.perf_counter() - t0

    # the plain backend, same compile settings as the server, one request at a time
    eng = QAOAEnergyEngine(device=device_index, max_width=29, max_slices=1024, order_trials=4,
                           cache_size=1)
    plain_lat, plain_edges, plain_err, n_plain = [], 0, 0.0, 0
    t0 = time.perf_counter()
    for (G, gamma, beta), batched in zip(reqs, stream):
        if time.perf_counter() - t0 > plain_budget_s:
            break
        if isinstance(batched, Exception):
            continue
        t = time.perf_counter()
        E = eng.energy_expectation(G, gamma, beta, path='plain')
        plain_lat.append((time.perf_counter() - t) * 1e3)
        plain_edges += G.number_of_edges()
        plain_err = max(plain_err, abs(E - batched.energy) / max(abs(batched.energy), 1e-30))
        n_plain += 1
    wall_plain = time.perf_counter() - t0
    plain = {'completed': n_plain, 'p50_ms': pct(plain_lat, 50), 'p95_ms': pct(plain_lat, 95),
             'p99_ms': pct(plain_lat, 99),
             'edge_terms_per_s': plain_edges / wall_plain if wall_plain > 0 else None,
             'wall_s': wall_plain, 'max_rel_diff_vs_batched': plain_err,
             'sample': 'the first admissible requests of the stream, in order, for about {:.0f} s'.format(
                 plain_budget_s)}

    def same(a, b):
        if isinstance(a, Exception) or isinstance(b, Exception):
            return isinstance(a, Exception) and isinstance(b, Exception)
        return a.energy == b.energy
    host = {'os_cpu_count': os.cpu_count(), 'available_cpus': _available_cpus()}
    return {'host_cpus': host,
            'workload': '{} requests: 3-regular or Erdos-Renyi (mean degree 3), N U[16,500], '
                        'p U[1,4], angles U[0,pi) (seed 0); Poisson arrivals at {} req/s '
                        '(seed 1); slicing from width 29, at most 1024 slices per edge, at most '
                        '{:.0e} algorithmic bytes per request; each server first answers 6 untimed '
                        'requests of the same distribution (seed 7)'.format(len(reqs), rate, budget),
            'continuous_batching': summarize(stream, wall_stream),
            'fifo_queue': summarize(fifo, wall_fifo),
            'batched_one_at_a_time': summarize(alone, wall_alone),
            'plain_one_at_a_time': plain,
            'same_energy_alone_and_in_mix': all(same(a, b) for a, b in zip(stream, alone))}


def oracle_error(eng, G, p):
    """Edge terms at the reference fixture's angles against its complex128
    values (the fixture holds every edge of the seed-0 workload graph)."""
    path = os.path.join(ROOT, 'tests', 'golden', 'qaoa_reference.json')
    try:
        with open(path) as f:
            w = json.load(f)['workloads']['cfg3']
    except (OSError, KeyError, ValueError):
        return None
    if [list(e) for e in G.edges()] != [list(e) for e in w['edges']] or len(w['gamma']) != p:
        return None
    terms = eng.edge_terms(G, w['gamma'], w['beta'])
    ref = np.array([complex(*t) for t in w['terms']])
    E = eng.energy_expectation(G, w['gamma'], w['beta'])
    return {'edge_terms': len(ref), 'max_abs_error': float(np.max(np.abs(terms - ref))),
            'mean_abs_error': float(np.mean(np.abs(terms - ref))),
            'energy_rel_error': abs(E - w['energy']) / abs(w['energy']),
            'oracle': 'complex128 reference values, tests/golden/qaoa_reference.json'}


# ------------------------------------------------------------------ plain backend by width
def plain_width_classes(device_index, reps=10, per_class=64):
    """The drop-in bucket kernel (qtb_bucket_c64, BucketBackend.process_bucket)
    per bucket output-width class, on the real bucket shapes of the 3-regular
    N=100 p=3 workload's plans (up to `per_class` buckets per width, random
    complex64 operands of their shapes, launched back to back), plus one
    24-variable bucket (64 MB in, 64 MB out) for the bandwidth-bound end.
    GB/s of algorithmic bytes 8 (sum of inputs + output)."""
    import ctypes
    import torch
    from qtensor_b200 import _lib
    from qtensor_b200.engine import QAOAEnergyEngine
    lib = _lib.lib()
    dev = torch.device('cuda', device_index)
    G2 = graphs.regular(100, seed=0)
    g, b = graphs.angles(3, seed=0)
    ex = QAOAEnergyEngine(device=device_index).compile(G2, 3, g, b).plan.export()
    ops, ins = ex['ops'], ex['ins']
    classes = {}
    for o in ops:
        classes.setdefault(int(o['u']) - int(o['sum']), []).append(o)
    gen = torch.Generator(device=dev).manual_seed(0)

    def time_buckets(descs, nbytes):
        stream = torch.cuda.current_stream(dev)
        for d, ptrs, out in descs:    # warm-up
            _lib.check(lib.qtb_bucket_c64(ctypes.byref(d), ptrs, out, ctypes.c_void_p(stream.cuda_stream)))
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(reps):
            for d, ptrs, out in descs:
                _lib.check(lib.qtb_bucket_c64(ctypes.byref(d), ptrs, out, ctypes.c_void_p(stream.cuda_stream)))
        e.record(stream)
        e.synchronize()
        ms = s.elapsed_time(e) / reps
        return {'buckets': len(descs), 'us_per_bucket': 1e3 * ms / len(descs),
                'gbs': nbytes / (ms / 1e3) / 1e9}

    def make(masks, n_vars, sum_first, keep):
        d = _lib.BucketDesc()
        d.n_inputs, d.n_vars, d.sum_first = len(masks), n_vars, sum_first
        bufs, nbytes = [], 0
        for i, m in enumerate(masks):
            d.masks[i] = m
            t = torch.randn(1 << bin(m).count('1'), dtype=torch.complex64, device=dev, generator=gen)
            bufs.append(t)
            nbytes += 8 * t.numel()
        out = torch.empty(1 << (n_vars - sum_first), dtype=torch.complex64, device=dev)
        nbytes += 8 * out.numel()
        keep.extend(bufs + [out])
        ptrs = (ctypes.c_void_p * len(masks))(*[t.data_ptr() for t in bufs])
        return (d, ptrs, ctypes.c_void_p(out.data_ptr())), nbytes

    result, keep = {}, []
    for w in sorted(classes):
        descs, nbytes = [], 0
        for o in classes[w][:per_class]:
            masks = [int(ins[int(o['in_begin']) + t]['mask']) for t in range(int(o['k']))]
            dsc, nb = make(masks, int(o['u']), int(o['sum']), keep)
            descs.append(dsc)
            nbytes += nb
        result['w%d' % w] = time_buckets(descs, nbytes)
    u = 24
    dsc, nb = make([((1 << u) - 1) & ~1, (1 << (u - 1)) | 0xfff, (1 << (u - 1)) | 1], u, 1, keep)
    result['bucket24'] = time_buckets([dsc], nb)
    return {'workload': 'bucket shapes of the 3-regular N=100 p=3 plans by output width (up to {} per '
                        'class, back to back, {} repetitions) and one 24-variable bucket; GB/s of '
                        'algorithmic bytes'.format(per_class, reps),
            'classes': result}


# ------------------------------------------------------------------ GPU arm
def measured_peak_hbm():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(path) as f:
            return float(json.load(f)['hbm_gbs']), 'measured'
    except (OSError, KeyError, ValueError):
        return 6650.0, 'fallback'


def profiled_traffic(key='dram_bytes_per_step'):
    """DRAM bytes (or, with key='warp_instructions_per_step', the executed
    warp-instructions) of the executor's launches per step, from the
    committed ncu summary, if any."""
    path = os.path.join(ROOT, 'profiles', 'network_kernel_cfg3.json')
    try:
        with open(path) as f:
            return json.load(f).get(key)
    except (OSError, ValueError):
        return None


def issue_roofline(kernel_ms, clk, device_index):
    """The executor's instruction-issue rate: ncu's warp-instructions per
    step over the live executor span, per SM and SM cycle at the median
    clock sampled during the timed region, against the 4 instructions an
    SM can issue per cycle (one per scheduler).  The executor keeps its
    intermediates in shared memory, so this, not HBM, is what bounds it."""
    import torch
    instr = profiled_traffic('warp_instructions_per_step')
    mhz = (clk or {}).get('sm_mhz')
    if not instr or not mhz or not kernel_ms:
        return None
    sms = torch.cuda.get_device_properties(device_index).multi_processor_count
    achieved = instr / (kernel_ms * 1e-3 * sms * mhz * 1e6)
    return {'achieved': achieved, 'peak': 4.0, 'unit': 'warp-instructions issued per SM cycle',
            'frac': achieved / 4.0, 'warp_instructions_per_step': instr, 'sms': sms, 'sm_mhz': mhz,
            'source': 'instruction count from ncu (profiles/network_kernel_cfg3.json), time live'}


def device_steps(eng, cg, G, p, angle_sets, flush, stream, warmup, steps):
    """Device-resident steps of a compiled graph: per step, the step's
    angles are checked on the host against the plan's angle-dependent
    simplifier decisions (qtb_plan_check_params; a plan that no longer holds
    is recompiled before the step, outside the events), copied device to
    device into the plan's angle buffer, and one captured contraction graph
    is replayed; CUDA events around each step, L2 flushed between steps.
    Returns (per-step ms, the compiled graph in use, angle-check record)."""
    import torch
    dev = cg.params.device
    params_dev = [torch.from_numpy(a).to(dev) for a in angle_sets]
    checks = {'steps_checked': 0, 'recompiled': 0}

    def ready(i):
        nonlocal cg
        checks['steps_checked'] += 1
        if cg.angle_checks and not cg.plan.params_valid(angle_sets[i]):
            cg = eng.compile(G, p, angle_sets[i][:p], angle_sets[i][p:])
            checks['recompiled'] += 1
        return cg.device_graph()

    for i in range(warmup):
        graph = ready(i)
        cg.params.copy_(params_dev[i])
        graph.replay()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for i in range(steps):
        graph = ready(warmup + i)
        flush.fill_(float(i))
        starts[i].record(stream)
        cg.params.copy_(params_dev[warmup + i])
        graph.replay()
        ends[i].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in zip(starts, ends)], cg, checks


def run_cfg4(device_index, flush, steps, warmup=3):
    """3-regular N=256 p=4 (seed 0, 384 edge terms): compile, error of every
    edge term against the complex128 reference fixture, device-resident
    edge terms/s, and how the networks split between the shared-memory
    executor (K3) and the wide waves (K4)."""
    import torch
    from qtensor_b200.engine import QAOAEnergyEngine
    with open(os.path.join(ROOT, 'tests', 'golden', 'qaoa_reference.json')) as f:
        w = json.load(f)['workloads']['cfg4']
    G = graphs.regular(256)
    assert [list(e) for e in G.edges()] == w['edges']
    eng = QAOAEnergyEngine(device=device_index)
    t0 = time.perf_counter()
    cg = eng.compile(G, 4, w['gamma'], w['beta'])
    compile_s = time.perf_counter() - t0
    terms = eng.edge_terms(G, w['gamma'], w['beta'])
    ref = np.array([complex(*t) for t in w['terms']])
    E = eng.energy_expectation(G, w['gamma'], w['beta'])
    angle_sets = [np.concatenate(graphs.angles(4, seed=400 + i)) for i in range(warmup + steps)]
    stream = torch.cuda.current_stream()
    step_ms, cg, checks = device_steps(eng, cg, G, 4, angle_sets, flush, stream, warmup, steps)
    ms = sum(step_ms) / steps
    stats = cg.stats()
    cfg = cg.plan.last_launch_config()
    wave_nets = sum(c[0] for c in cfg if c[3] & 4)
    return {'workload': '3-regular N=256 (seed 0), p=4, default composer, native order; '
                        '384 edge-term networks per step; no slicing needed (widths below 29)',
            'edge_terms_per_s': stats['edges'] / (ms / 1e3), 'ms_per_step': ms, 'steps': steps,
            'compile_s': compile_s, 'width_max': stats['width_max'], 'networks': stats['networks'],
            'alg_bytes_per_step': stats['alg_bytes'],
            'alg_gbs_per_step_time': stats['alg_bytes'] / (ms / 1e3) / 1e9,
            'networks_shared_memory_executor': stats['networks'] - wave_nets,
            'networks_wide_waves': wave_nets,
            'launch_classes': [{'networks': c[0], 'threads': c[1], 'smem_bytes': c[2], 'flags': c[3]}
                               for c in cfg],
            'max_abs_error_vs_oracle': float(np.max(np.abs(terms - ref))),
            'energy_rel_error': abs(E - w['energy']) / abs(w['energy']),
            'angle_checks': checks}


def run_reference_order(G, p, device_index, flush, steps, warmup=3):
    """The headline workload with QTensor's own lightcone numbering and greedy
    elimination order (ordering='reference'), so that the order search's
    share of the speed-up is visible."""
    import torch
    from qtensor_b200.engine import QAOAEnergyEngine
    eng = QAOAEnergyEngine(ordering='reference', device=device_index)
    g0, b0 = graphs.angles(p, seed=0)
    t0 = time.perf_counter()
    cg = eng.compile(G, p, g0, b0)
    compile_s = time.perf_counter() - t0
    angle_sets = [np.concatenate(graphs.angles(p, seed=100 + i)) for i in range(warmup + steps)]
    step_ms, cg, checks = device_steps(eng, cg, G, p, angle_sets, flush, torch.cuda.current_stream(),
                                       warmup, steps)
    ms = sum(step_ms) / steps
    stats = cg.stats()
    return {'edge_terms_per_s': stats['edges'] / (ms / 1e3), 'ms_per_step': ms, 'steps': steps,
            'compile_s': compile_s, 'width_max': stats['width_max'],
            'alg_bytes_per_step': stats['alg_bytes'], 'angle_checks': checks}


def run_dropin(device_index):
    """The drop-in path as the reference drives it: every backend call the
    reference's QAOAQtreeSimulator made with its NumpyBackend (recorded in
    tests/golden/dropin_trace.json) replayed into B200Backend -- one
    qtb_bucket_c64 launch per process_bucket -- timed per edge term."""
    import torch
    import dropin_replay
    from qtensor_b200.backend import B200Backend
    be = B200Backend(device=device_index)
    out = {}
    for name, w in dropin_replay.load().items():
        inputs = [dropin_replay.edge_inputs(rec) for rec in w['edges']]
        dropin_replay.replay_edge(be, w['edges'][0], inputs[0])     # warm-up
        torch.cuda.synchronize()
        err = 0.0
        t0 = time.perf_counter()
        for rec, inp in zip(w['edges'], inputs):
            amp, _ = dropin_replay.replay_edge(be, rec, inp)
            err = max(err, float(np.max(np.abs(amp - [complex(*z) for z in rec['amplitude']]))))
        dt = time.perf_counter() - t0
        calls = sum(len(r['calls']) for r in w['edges'])
        out[name] = {'edges': len(w['edges']), 'process_bucket_calls': calls,
                     'edge_terms_per_s': len(w['edges']) / dt, 'us_per_process_bucket': 1e6 * dt / calls,
                     'max_abs_error_vs_recorded': err}
    out['what'] = ("the reference QAOAQtreeSimulator's recorded get_sliced_buckets / process_bucket / "
                   'get_result_data calls replayed into B200Backend (host Python per call, one bucket '
                   'kernel launch per process_bucket, result read back per edge)')
    return out


def measured_peak_tflops():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d['bf16_tflops']), 'measured (dense bf16 cuBLAS burst)'
    except (OSError, KeyError, ValueError):
        return 1590.0, 'fallback'


def run_tensor_core_contract(device_index, reps=5):
    """The reference's merged-index contraction C[f,m,n] = sum_k A[k,f,m]
    B[k,f,n] (CMKLExtendedBackend's mkl_contract_sum) on a GEMM-shaped
    workload, K = 1024, F = 2, M = N = 1024: the tcgen05 path (3xTF32
    products, FP32 accumulation) against the CUDA-core path, with the
    useful complex flops 8 F M N K per call and the error of 16 sampled
    output rows against complex128 (numpy, on the host)."""
    import torch
    from qtensor_b200 import tcontract
    dev = torch.device('cuda', device_index)
    K, F, M, N = 1024, 2, 1024, 1024
    rng = np.random.default_rng(7)
    A = (rng.standard_normal((K, F, M)) + 1j * rng.standard_normal((K, F, M))).astype(np.complex64)
    B = (rng.standard_normal((K, F, N)) + 1j * rng.standard_normal((K, F, N))).astype(np.complex64)
    a, b = torch.from_numpy(A).to(dev), torch.from_numpy(B).to(dev)
    out = {}
    flops = 8.0 * F * M * N * K
    for mode in ('tensor', 'simt'):
        c = torch.empty((F, M, N), dtype=torch.complex64, device=dev)
        scratch = torch.empty(tcontract.contract_sum_scratch_bytes(K, F, M, N, mode), dtype=torch.uint8, device=dev)
        tcontract.mkl_contract_sum(a, b, c, mode=mode, scratch=scratch)     # warm-up
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            tcontract.mkl_contract_sum(a, b, c, mode=mode, scratch=scratch)
        e.record()
        e.synchronize()
        ms = s.elapsed_time(e) / reps
        status = int(scratch[:4].view(torch.int32).item())
        rows = rng.choice(M, 16, replace=False)
        got = c.cpu().numpy()
        ref = np.einsum('kfm,kfn->fmn', A[:, :, rows].astype(np.complex128), B.astype(np.complex128))
        err = float(np.max(np.abs(got[:, rows, :] - ref)) / np.max(np.abs(ref)))
        out[mode] = {'ms': ms, 'useful_tflops': flops / (ms / 1e3) / 1e12, 'status': status,
                     'max_rel_error_vs_complex128': err}
    peak, source = measured_peak_tflops()
    out['tensor']['frac_of_peak'] = out['tensor']['useful_tflops'] / peak
    out['peak_tflops'] = peak
    out['peak_source'] = source
    out['tensor_over_simt'] = out['simt']['ms'] / out['tensor']['ms']
    out['workload'] = ('C[f,m,n] = sum_k A[k,f,m] B[k,f,n], K=1024 F=2 M=N=1024 complex64 (includes the '
                       'TF32 hi/lo split pre-pass); useful flops 8 F M N K; the 3xTF32 emulation runs 12 real '
                       'MMA passes per complex product, so the useful rate is at most 1/3 of the TF32 rate')
    return out


def run_sharded(args, dev, local, rank, world):
    """One Erdos-Renyi graph (mean degree 3, p=3) sharded over the ranks by
    longest processing time on the plans' flops: each rank contracts its
    share and one NCCL all-reduce of fp64 shares gives every rank the
    energy (DistributedQAOAEnergy).  Timed per energy with CUDA events on
    every rank, max over ranks."""
    import torch
    import torch.distributed as dist
    from qtensor_b200.distributed import DistributedQAOAEnergy
    G = graphs.erdos_renyi(args.shard_nodes, seed=24323709)
    p = 3
    denergy = DistributedQAOAEnergy(lpt=True, device=local)
    for i in range(args.warmup):
        denergy.energy_expectation(G, *graphs.angles(p, seed=500 + i))
    torch.cuda.synchronize()
    dist.barrier()
    stream = torch.cuda.current_stream(dev)
    total_ms, energies = 0.0, []
    for i in range(args.steps):
        g, b = graphs.angles(p, seed=600 + i)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        energies.append(denergy.energy_expectation(G, g, b))
        e.record(stream)
        e.synchronize()
        total_ms += s.elapsed_time(e)
    dist.barrier()
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = t.item() / args.steps
    n_edges = G.number_of_edges()
    if rank == 0:
        print(json.dumps({
            'metric': 'QAOA edge terms/s (Erdos-Renyi N={} p=3, edges sharded over ranks)'.format(args.shard_nodes),
            'value': n_edges / (ms / 1e3), 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True, 'scaling': 'strong',
            'vs_baseline': None, 'dtype': 'c64', 'data': 'synthetic', 'impl': 'b200', 'mode': 'shard',
            'config': {'workload': 'one Erdos-Renyi graph N={} (seed 24323709), p=3, {} edges; LPT '
                                   'shards by plan flops; one NCCL all-reduce per energy'.format(
                                       args.shard_nodes, n_edges)},
            'energy_first_step': energies[0] if energies else None}), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def run_b200(args):
    rank, world, local = dist_env()
    G = graphs.regular(args.nodes, seed=rank)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # timed before CUDA is initialised, so the pool may fork
        n_sample = cpu_sample_edges(G.number_of_edges())
        rate, cores, dt = cpu_reference(G, args.p, n_sample, seed=0, start_method='fork')
        n_one = min(32, G.number_of_edges())
        rate1, dt1 = cpu_single_process(G, args.p, n_one, seed=0)
        cpu = {'value': rate, 'unit': UNIT, 'cores': cores, 'kind': 'port',
               'sample': '{} of {} edges of the workload through the oracle port of '
                         'energy_expectation_parallel (NumpyBackend einsum, complex128), '
                         '{} processes, {:.1f} s'.format(n_sample, G.number_of_edges(), cores, dt),
               'single_process': {'value': rate1, 'unit': UNIT,
                                  'sample': 'the first {} edges, serial edge loop, {:.1f} s'.format(n_one, dt1)}}

    import torch
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=120), device_id=dev)
        pg = dist
        if args.shard:
            return run_sharded(args, dev, local, rank, world)
    # nvidia-smi takes a moment to start; launch it before the compile so
    # its samples cover warm-up and the timed steps
    clocks = ClockSampler(local)
    clocks.start()

    from qtensor_b200.engine import QAOAEnergyEngine
    eng = QAOAEnergyEngine(composer='default', ordering='native', device=local)
    p = args.p
    gamma0, beta0 = graphs.angles(p, seed=0)
    t0 = time.perf_counter()
    cg = eng.compile(G, p, gamma0, beta0)
    compile_s = time.perf_counter() - t0
    # the rest of a cold public call: autotune on the first launch, graph
    # capture, one replay (compile + this = the cold end-to-end time)
    t0 = time.perf_counter()
    eng.energy_expectation(G, gamma0, beta0)
    first_call_s = time.perf_counter() - t0
    stats = cg.stats()
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    angle_sets = [np.concatenate(graphs.angles(p, seed=100 + i)) for i in range(args.warmup + args.steps)]

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()

    # ---- device-resident steps (clock samples cover warm-up and timed steps)
    barrier()
    step_ms, cg, angle_checks = device_steps(eng, cg, G, p, angle_sets, flush, stream, args.warmup,
                                             args.steps)
    barrier()
    # the executor alone: external timing events captured around the class
    # launches (fork to join) inside a graph, replayed once per step
    ev_a = torch.cuda.Event(enable_timing=True, external=True)
    ev_b = torch.cuda.Event(enable_timing=True, external=True)
    tgraph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(tgraph):
        ev_a.record()
        cg.launch(stream=torch.cuda.current_stream(dev))
        ev_b.record()
    n_classes = len(cg.plan.last_launch_config())
    kernel_ms = 0.0
    params_dev = [torch.from_numpy(a).to(dev) for a in angle_sets]
    for i in range(args.steps):
        flush.fill_(float(i))
        cg.params.copy_(params_dev[args.warmup + i])
        tgraph.replay()
        ev_b.synchronize()
        kernel_ms += ev_a.elapsed_time(ev_b)
    kernel_launches = n_classes * args.steps
    del tgraph
    status = cg.plan.device_status()
    if status:
        raise RuntimeError('device status {:#x}'.format(status))

    # ---- end-to-end through the public API (host angles in, energy out)
    e2e_ms = []
    for i in range(args.warmup):
        eng.energy_expectation(G, *graphs.angles(p, seed=200 + i))
    barrier()
    for i in range(args.steps):
        gamma, beta = graphs.angles(p, seed=300 + i)
        flush.fill_(float(i))
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        eng.energy_expectation(G, gamma, beta)
        e.record(stream)
        e.synchronize()
        e2e_ms.append(s.elapsed_time(e))
    barrier()
    clk = clocks.stop()

    # ---- the plain path: one bucket-kernel launch per bucket over the same
    # plans (the drop-in backend's kernel), a few steps
    plain_steps = args.plain_steps
    if plain_steps:
        cg.params.copy_(params_dev[0])
        cg.launch_plain()
    plain_ms = []
    for i in range(plain_steps):
        flush.fill_(float(i))
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        cg.params.copy_(params_dev[args.warmup + i])
        cg.launch_plain()
        e.record(stream)
        e.synchronize()
        plain_ms.append(s.elapsed_time(e))
    plain_ms_step = sum(plain_ms) / plain_steps if plain_steps else float('nan')

    errors = oracle_error(eng, G, p) if rank == 0 else None
    extra = rank == 0 and world == 1
    plain_widths = plain_width_classes(local) if extra and args.plain_steps > 0 else None
    cfg4 = run_cfg4(local, flush, args.cfg4_steps) if extra and args.cfg4_steps > 0 else None
    ref_order = (run_reference_order(G, p, local, flush, args.reference_order_steps)
                 if extra and args.reference_order_steps > 0 else None)
    dropin = run_dropin(local) if extra and not args.no_dropin else None
    tc_contract = run_tensor_core_contract(local) if extra and not args.no_tensor_core else None
    serving = None
    if extra and args.serving_requests > 0:
        serving = run_serving(args.serving_requests, args.serving_rate, local)
    if extra and args.serving_saturate > 0:
        serving = dict(serving or {})
        serving['saturated'] = run_serving_saturated(args.serving_saturate, args.serving_saturate_rate, local)

    total_ms = sum(step_ms)
    e2e_total = sum(e2e_ms)
    if pg:
        t = torch.tensor([total_ms, e2e_total], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms, e2e_total = t.tolist()
    ms_per_step = total_ms / args.steps
    value = world * stats['edges'] / (ms_per_step / 1e3)
    e2e_value = world * stats['edges'] / (e2e_total / args.steps / 1e3)
    # the size classes of one step run concurrently (forked streams): the
    # executor's span per step, fork to join, is the launch duration used
    kernel_step_ms = kernel_ms / args.steps
    launches_per_step = kernel_launches / args.steps
    peak, peak_kind = measured_peak_hbm()
    achieved = stats['alg_bytes'] / (kernel_step_ms / 1e3) / 1e9
    cold_e2e_s = compile_s + first_call_s
    cold_rate = stats['edges'] / cold_e2e_s
    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms_per_step,
            'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': value / PUBLISHED_TERMS_PER_S, 'dtype': 'c64', 'data': 'synthetic',
            'impl': 'b200',
            'config': dict(WORKLOAD, l2='flushed between steps (256 MiB write outside the events)',
                           parallelism='one graph per rank' if world > 1 else 'single GPU',
                           width_max=stats['width_max'], ops_per_step=stats['ops'],
                           compile_s=compile_s, first_call_s=first_call_s,
                           cold_e2e_s=cold_e2e_s, cold_e2e_terms_per_s=cold_rate,
                           cold_ratio_vs_cpu_baseline=(cold_rate / cpu['value']) if cpu else None,
                           alg_bytes_per_step=stats['alg_bytes'],
                           angle_checks=angle_checks,
                           launch_classes=[{'networks': c[0], 'threads': c[1], 'smem_bytes': c[2],
                                            'smem_arena': bool(c[3] & 1), 'persistent': bool(c[3] & 2),
                                            'warp_queue': bool(c[3] & 16)}
                                           for c in cg.plan.last_launch_config()],
                           alg_flops_per_step=stats['alg_flops']),
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak, 'traffic': profiled_traffic(),
                         'kernel': 'qtb_network_kernel / qtb_warp_network_kernel', 'peak_source': peak_kind,
                         'kernel_ms_per_step': kernel_step_ms,
                         'class_launches_per_step': launches_per_step,
                         'alg_bytes_per_step': stats['alg_bytes'],
                         'issue': issue_roofline(kernel_step_ms, clk, local)},
            'cpu_baseline': cpu,
            'e2e': {'value': e2e_value, 'unit': UNIT, 'h2d_bytes_per_step': 8 * 2 * p,
                    'd2h_bytes_per_step': 8, 'ms_per_step': e2e_total / args.steps},
            'clocks': clk,
            'error_vs_oracle': errors,
            'reference_order': ref_order,
            'cfg4': cfg4,
            'dropin': dropin,
            'tensor_core_contract': tc_contract,
            'plain_by_width': plain_widths,
            'plain': None if not plain_steps else {'value': stats['edges'] / (plain_ms_step / 1e3), 'unit': UNIT,
                      'ms_per_step': plain_ms_step, 'steps': plain_steps,
                      'bucket_launches_per_step': stats['ops'],
                      'what': 'same plans, one qtb_bucket_kernel launch per bucket (the '
                              'drop-in process_bucket kernel), networks in sequence, '
                              'intermediates in global memory, complex64',
                      'batched_over_plain': value / (world * stats['edges'] / (plain_ms_step / 1e3))},
            'serving': serving,
            # every kernel of a step is an executor launch (gate table and
            # energy reduction are fused into it)
            'gpu_launches': int(kernel_launches),
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def main():
    args = parse()
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_b200(args)


if __name__ == '__main__':
    main()
