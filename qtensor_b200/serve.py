"""Continuous-batching QAOA energy server on one GPU.

Requests ``(G, gamma, beta)`` arrive at any time (``submit`` returns a
``concurrent.futures.Future``).  Each request's edge networks are compiled on
host worker threads (C++ plan compiler, native lightcones, slicing above
``max_width``), then admitted to the GPU when its plan memory fits the
device budget and a stream slot is free.  Admitted requests run on their own
CUDA stream, so a request that arrives while others are on the GPU starts as
soon as it is admitted and its kernels overlap theirs.  Plans, gate tensors
and partial sums stay on the device; one 8-byte energy per request is read
back.  A request that fails (compile error, over budget, device status)
fails only its own future.

The energy of a request is the value of ``QAOASimulator.energy_expectation``
(qtensor/QAOASimulator.py:44-66) for its graph and angles.
"""
import collections
import queue
import threading
import time
from concurrent.futures import Future, ThreadPoolExecutor

import numpy as np
import torch

from . import _lib
from .lightcone import composer_id
from .plan import NetworkPlan, graph_csr


class Result:
    """Energy of one request with its timeline (host clock, seconds):
    submitted -> compiled (plan built on a host worker) -> admitted (launched
    on a stream) -> finished (energy on the host)."""
    __slots__ = ('energy', 'edges', 'networks', 'submitted', 'admitted', 'finished', 'compiled')

    def __init__(self, energy, edges, networks, submitted, admitted, finished, compiled=None):
        self.energy = energy
        self.edges = edges
        self.networks = networks
        self.submitted = submitted
        self.admitted = admitted
        self.finished = finished
        self.compiled = admitted if compiled is None else compiled

    @property
    def latency(self):
        return self.finished - self.submitted

    @property
    def compile_s(self):
        """Waiting for a compile worker plus compiling."""
        return self.compiled - self.submitted

    @property
    def wait_s(self):
        """Compiled, waiting for memory or a stream slot."""
        return self.admitted - self.compiled

    @property
    def gpu_s(self):
        """Admitted until the energy reached the host."""
        return self.finished - self.admitted


class RequestTooLarge(RuntimeError):
    """A request whose contraction work exceeds the server's budget."""


class _Compiled:
    __slots__ = ('future', 'plan', 'params', 'n_edges', 'n_networks', 'bytes', 'scratch', 'submitted',
                 'compiled')


class _Inflight:
    __slots__ = ('job', 'slot', 'event', 'energy_host', 'buffers', 'admitted')


class AdmissionControl:
    """Device-memory budget and stream slots of the server (host logic)."""

    def __init__(self, budget_bytes, slots):
        self.budget = int(budget_bytes)
        self.used = 0
        self.free_slots = list(range(slots))

    def fits_ever(self, nbytes):
        return nbytes <= self.budget

    def try_admit(self, nbytes):
        """A slot index if the request fits now, else None."""
        if not self.free_slots or self.used + nbytes > self.budget:
            return None
        self.used += nbytes
        return self.free_slots.pop(0)

    def release(self, slot, nbytes):
        self.used -= nbytes
        self.free_slots.append(slot)
        self.free_slots.sort()


class QAOAServer:
    """Continuous-batching energy server.

    n_streams: requests in flight on the GPU at once; memory_budget: bytes of
    device memory the in-flight requests may hold (default: three quarters
    of the device's memory); max_width: networks whose width (best of the
    greedy and minimum-fill orders) reaches it are sliced, into at most
    max_slices networks per edge.  The default 29 keeps every unsliced
    network's largest tensor at 2^28 complex64 elements (2 GiB) and its
    arena below 16 GiB, so only circuits that do not fit HBM are sliced.  A
    request that would need more slices fails alone and fast: its lightcones
    are wider than any exact contraction on one GPU can hold (the reference
    would have to allocate tensors of that width too).  max_request_bytes:
    a request whose plans move more algorithmic bytes than this (the sum
    over its buckets of inputs read plus output written) fails at compile
    time instead of holding the GPU for minutes; None admits any.
    order_trials: randomized greedy orders per network (plus the minimum-fill
    candidates they bring), fewer than the engine's 16 because a request's
    compile is on its latency path.  compile_workers: host threads compiling
    requests concurrently, each with compile_threads C++ threads (default:
    its share of the CPUs the process may use).  wave_ctas_per_sm: resident
    CTAs per SM of a wide request's whole-GPU waves (1 leaves half of every
    SM to the other requests' kernels while a wide request runs; 0 lets
    the waves take whole SMs).  Every request's persistent launches claim
    all their networks from their queues (the engine's dynamic_claims): with
    concurrent requests holding SMs, a CTA that starts late takes whatever
    network is left rather than one fixed in advance."""

    def __init__(self, device=None, n_streams=4, memory_budget=None, max_width=29,
                 max_slices=1024, composer='default', order_trials=4, compile_workers=2,
                 compile_threads=0, max_request_bytes=None, wave_ctas_per_sm=1):
        if not torch.cuda.is_available():
            raise RuntimeError('QAOAServer needs a CUDA device; there is no CPU fallback')
        self.device = torch.device('cuda', torch.cuda.current_device() if device is None else device)
        self.cid = composer_id(composer)
        self.max_width = max_width
        self.max_slices = max_slices
        self.order_trials = order_trials
        # the compile workers share the CPUs the process may use
        self.compile_threads = compile_threads or max(1, _lib.available_cpus() // max(1, compile_workers))
        self.wave_ctas_per_sm = wave_ctas_per_sm
        self.max_request_bytes = max_request_bytes
        _lib.check(_lib.lib().qtb_init(self.device.index))
        if memory_budget is None:
            memory_budget = torch.cuda.get_device_properties(self.device).total_memory * 3 // 4
        self.admission = AdmissionControl(memory_budget, n_streams)
        self.streams = [torch.cuda.Stream(self.device) for _ in range(n_streams)]
        self._compile_pool = ThreadPoolExecutor(max_workers=compile_workers)
        self._ready = queue.Queue()          # compiled requests, arrival order
        self._stop = threading.Event()
        self._retired = []                   # finished plans awaiting release (dispatcher only)
        self._dispatcher = threading.Thread(target=self._dispatch_loop, daemon=True)
        self._dispatcher.start()
        self.stats = collections.Counter()

    # ------------------------------------------------------------ client
    def submit(self, G, gamma, beta):
        """Queue an energy request; the future resolves to a ``Result``."""
        fut = Future()
        submitted = time.perf_counter()
        self._compile_pool.submit(self._compile, fut, G, list(gamma), list(beta), submitted)
        return fut

    def energy(self, G, gamma, beta, timeout=None):
        return self.submit(G, gamma, beta).result(timeout).energy

    def close(self):
        self._compile_pool.shutdown(wait=True)
        self._stop.set()
        self._ready.put(None)
        self._dispatcher.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ compile
    def _compile(self, fut, G, gamma, beta, submitted):
        try:
            if len(gamma) != len(beta):
                raise ValueError('gamma and beta must have the same length')
            p = len(gamma)
            params = np.concatenate([np.asarray(gamma, np.float64), np.asarray(beta, np.float64)])
            csr = graph_csr(G)
            index = {v: i for i, v in enumerate(csr[0])}
            edges = np.array([(index[a], index[b]) for a, b in G.edges()], dtype=np.int32)
            if len(edges) == 0:
                # an empty sum of edge terms, as the reference computes it
                # (QAOASimulator.py:27-41): nothing to run on the GPU
                now = time.perf_counter()
                self.stats['done'] += 1
                fut.set_result(Result(0.0, 0, 0, submitted, now, now))
                return
            torch.cuda.set_device(self.device)
            plan = NetworkPlan(2 * p)
            plan.set_order_trials(self.order_trials)
            plan.set_max_width(self.max_width, self.max_slices)
            plan.set_wave_ctas_per_sm(self.wave_ctas_per_sm)
            plan.set_dynamic_claims(True)
            plan.add_lightcones(csr, edges, p, self.cid, params, self.compile_threads)
            if self.max_request_bytes is not None:
                work = sum(plan.info(i)['alg_bytes'] for i in range(len(plan)))
                if work > self.max_request_bytes:
                    plan.close()
                    raise RequestTooLarge('request moves {:.3g} bytes in its contractions, over the '
                                          'server\'s budget of {:.3g}'.format(work, self.max_request_bytes))
            job = _Compiled()
            job.future, job.plan, job.params = fut, plan, params
            job.n_edges, job.n_networks = len(edges), len(plan)
            job.submitted = submitted
            # plan images + run buffers (terms, energy, params) + scratch (the
            # arenas of wide networks), all known before anything is allocated
            job.scratch = plan.scratch_bytes(0, job.n_networks)
            job.bytes = plan.device_bytes() + job.scratch + 8 * job.n_networks + 64 + 8 * len(params)
            job.compiled = time.perf_counter()
            self._ready.put(job)
        except Exception as exc:     # noqa: BLE001 - the request fails alone
            self.stats['failed'] += 1
            fut.set_exception(exc)

    # ------------------------------------------------------------ GPU side
    def _launch(self, job, slot):
        stream = self.streams[slot]
        with torch.cuda.stream(stream):
            job.plan.upload()
            scratch_bytes = job.scratch
            buffers = {
                'params': torch.from_numpy(job.params).to(self.device, non_blocking=False),
                'terms': torch.empty(job.n_networks, dtype=torch.complex64, device=self.device),
                'energy': torch.empty(1, dtype=torch.float64, device=self.device),
                'scratch': (torch.empty(scratch_bytes, dtype=torch.uint8, device=self.device)
                            if scratch_bytes else None),
            }
            job.plan.run(0, job.n_networks, buffers['params'], buffers['terms'], buffers['energy'],
                         buffers['scratch'], stream.cuda_stream)
            host = torch.empty(1, dtype=torch.float64, pin_memory=True)
            host.copy_(buffers['energy'], non_blocking=True)
            event = torch.cuda.Event()
            event.record(stream)
        fl = _Inflight()
        fl.job, fl.slot, fl.event, fl.energy_host, fl.buffers = job, slot, event, host, buffers
        fl.admitted = time.perf_counter()
        return fl

    def _finish(self, fl):
        job = fl.job
        self.admission.release(fl.slot, job.bytes)
        try:
            status = job.plan.device_status()
            if status:
                raise _lib.QtbError(_lib.QTB_ERR_DEVICE, 'device status word {:#x}'.format(status))
            res = Result(float(fl.energy_host.numpy()[0]), job.n_edges, job.n_networks,
                         job.submitted, fl.admitted, time.perf_counter(), job.compiled)
            self.stats['done'] += 1
            job.future.set_result(res)
        except Exception as exc:     # noqa: BLE001
            self.stats['failed'] += 1
            job.future.set_exception(exc)
        finally:
            # freeing device memory synchronises the whole device, so finished
            # plans are released while the GPU has no request in flight (or
            # in batches), not while other requests' kernels run
            self._retired.append(job.plan)

    def _dispatch_loop(self):
        torch.cuda.set_device(self.device)
        waiting = collections.deque()      # compiled, not yet admitted (FIFO)
        inflight = []
        done_input = False
        while True:
            # take newly compiled requests without blocking while work is in flight
            block = not inflight and not waiting and not done_input
            try:
                item = self._ready.get(block=block, timeout=None if block else 0)
                while True:
                    if item is None:
                        done_input = True
                    else:
                        waiting.append(item)
                    item = self._ready.get_nowait()
            except queue.Empty:
                pass
            # admit in arrival order while memory and slots allow
            while waiting:
                job = waiting[0]
                if not self.admission.fits_ever(job.bytes):
                    waiting.popleft()
                    self.stats['rejected'] += 1
                    job.plan.close()
                    job.future.set_exception(MemoryError(
                        'request needs {} bytes of device memory, budget {}'.format(
                            job.bytes, self.admission.budget)))
                    continue
                slot = self.admission.try_admit(job.bytes)
                if slot is None:
                    break
                waiting.popleft()
                try:
                    inflight.append(self._launch(job, slot))
                except Exception as exc:     # noqa: BLE001
                    self.admission.release(slot, job.bytes)
                    self.stats['failed'] += 1
                    job.plan.close()
                    job.future.set_exception(exc)
            # retire finished requests
            still = []
            for fl in inflight:
                if fl.event.query():
                    self._finish(fl)
                else:
                    still.append(fl)
            inflight = still
            if self._retired and (not inflight or len(self._retired) >= 32):
                for plan in self._retired:
                    plan.close()
                self._retired = []
            if done_input and not inflight and not waiting:
                return
            if inflight:
                time.sleep(20e-6)
