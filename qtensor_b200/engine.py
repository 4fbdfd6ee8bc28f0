"""Batched QAOA MaxCut energies on one B200.

``QAOAEnergyEngine.energy_expectation(G, gamma, beta)`` has the signature and
meaning of ``QAOASimulator.energy_expectation`` (qtensor/QAOASimulator.py:44-66):
the sum over edges of ``<psi| Z_u Z_v |psi>`` post-processed to the expected
cut ``(|E| - Re sum) / 2`` (qtensor/QAOASimulator.py:27-41).

Every edge's lightcone network is compiled once per (graph, p, composer,
ordering) by the C++ plan compiler and kept on the device; a call uploads
the 2p angles, generates the gate tensors on the device, contracts all edge
networks (one CTA per network, intermediates in shared memory) and reduces
the edge terms in fp64 -- one CUDA-graph replay, one 8-byte read-back.
"""
import ctypes
import hashlib
import threading
import weakref

import numpy as np
import torch

from . import _lib
from .lightcone import composer_id, reference_lightcone, simplify_passes
from .plan import NetworkPlan, graph_csr


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError('qtensor_b200 needs a CUDA device; there is no CPU fallback')


def graph_key(G, p, composer, ordering, trials=0, slicing=(0, 0)):
    h = hashlib.sha1()
    h.update(repr((p, composer, ordering, trials, slicing, G.number_of_nodes())).encode())
    h.update(repr(list(G.nodes())).encode())
    h.update(repr(list(G.edges())).encode())
    return h.hexdigest()


class CompiledGraph:
    """Device-resident plan of all edge networks of one graph."""

    def __init__(self, plan, edges, p, composer, device):
        self.plan = plan
        self.edges = edges
        self.p = p
        self.composer = composer
        self.n_edges = len(edges)
        self.n_networks = len(plan)
        self.device = device
        # networks of one edge (its slices) are contiguous and share a group
        self.groups = plan.groups()
        self.terms = torch.empty(self.n_networks, dtype=torch.complex64, device=device)
        self.energy = torch.empty(1, dtype=torch.float64, device=device)
        self.params = torch.empty(2 * p, dtype=torch.float64, device=device)
        nbytes = plan.scratch_bytes(0, self.n_networks)
        self.scratch = (torch.empty(max(nbytes, 8), dtype=torch.uint8, device=device)
                        if nbytes else None)
        self._infos = None
        self._plain_scratch = None
        # simplifier decisions that hold only for some angles (rechecked per call)
        self.angle_checks = any(i['angle_specific'] for i in self.infos)
        # host side of the captured call: pinned angles in, pinned energy out
        self.host_params = torch.zeros(2 * p, dtype=torch.float64, pin_memory=True)
        self.host_energy = torch.zeros(1, dtype=torch.float64, pin_memory=True)
        self._graph = None

    @property
    def infos(self):
        if self._infos is None:
            self._infos = self.plan.infos()
        return self._infos

    def stats(self):
        infos = self.infos
        widths = [i['treewidth'] for i in infos]
        return {
            'edges': self.n_edges,
            'networks': self.n_networks,
            'width_max': max(widths), 'width_mean': float(np.mean(widths)),
            'ops': int(sum(i['n_ops'] for i in infos)),
            'phases_max': max(i['n_phases'] for i in infos),
            'arena_max_bytes': 8 * max(i['arena_elems'] for i in infos),
            'alg_bytes': float(sum(i['alg_bytes'] for i in infos)),
            'alg_flops': float(sum(i['alg_flops'] for i in infos)),
            'ref_flops': float(sum(i['ref_flops'] for i in infos)),
            'angle_specific': int(sum(i['angle_specific'] for i in infos)),
        }

    def launch(self, params_dev=None, stream=None):
        """Contract all edge networks asynchronously; energy lands in ``self.energy``."""
        stream = torch.cuda.current_stream(self.device) if stream is None else stream
        self.plan.run(0, self.n_networks, self.params if params_dev is None else params_dev,
                      self.terms, self.energy, self.scratch, stream.cuda_stream)

    def launch_plain(self, params_dev=None, stream=None):
        """The plain path, asynchronously: one bucket-kernel launch per bucket
        (the drop-in backend's process_bucket), networks in sequence,
        intermediates in global memory; results in ``self.terms`` and
        ``self.energy`` as with ``launch``."""
        stream = torch.cuda.current_stream(self.device) if stream is None else stream
        if self._plain_scratch is None:
            nbytes = self.plan.plain_scratch_bytes(0, self.n_networks)
            self._plain_scratch = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=self.device)
        self.plan.run_plain(0, self.n_networks, self.params if params_dev is None else params_dev,
                            self.terms, self.energy, self._plain_scratch, stream.cuda_stream)

    def edge_terms(self):
        """Per-edge amplitudes of the last run (slices summed), complex128."""
        vals = self.terms.cpu().numpy().astype(np.complex128)
        out = np.zeros(self.n_edges, dtype=np.complex128)
        np.add.at(out, self.groups - self.groups[0], vals)
        return out

    def _host_mapped(self, t):
        """Device pointer of a pinned host tensor, or None when the device
        cannot map it."""
        dev = ctypes.c_void_p()
        if _lib.lib().qtb_host_device_pointer(ctypes.c_void_p(t.data_ptr()), ctypes.byref(dev)) != 0:
            return None
        return dev.value

    def _capture(self):
        """CUDA graph of one call: pinned angles -> device, gate table,
        executor classes (forked streams), energy -> pinned host.  The angles
        are copied by a kernel that reads the pinned buffer through its
        device mapping, and the energy is written by the executor straight
        into the pinned result buffer: a graph without copy nodes (each cost
        several microseconds of a call of about fifty).  Without a mapping,
        copy nodes do the same."""
        lib = _lib.lib()
        with torch.cuda.device(self.device):
            self.launch()                      # builds the run's job arrays outside capture
            torch.cuda.synchronize(self.device)
            h_params, h_energy = self._host_mapped(self.host_params), self._host_mapped(self.host_energy)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                stream = torch.cuda.current_stream(self.device)
                if h_params is not None and h_energy is not None:
                    _lib.check(lib.qtb_copy_c(ctypes.c_void_p(self.params.data_ptr()), ctypes.c_void_p(h_params),
                                              8 * self.params.numel(), ctypes.c_void_p(stream.cuda_stream)))
                    self.plan.run(0, self.n_networks, self.params, self.terms, h_energy,
                                  self.scratch, stream.cuda_stream)
                else:
                    self.params.copy_(self.host_params, non_blocking=True)
                    self.launch(stream=stream)
                    self.host_energy.copy_(self.energy, non_blocking=True)
            self._graph = graph

    def device_graph(self):
        """CUDA graph of one contraction from the device-resident angles in
        ``self.params`` (no host copies); energy lands in ``self.energy``."""
        if getattr(self, '_dgraph', None) is None:
            with torch.cuda.device(self.device):
                self.launch()
                torch.cuda.synchronize(self.device)
                graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(graph):
                    self.launch(stream=torch.cuda.current_stream(self.device))
                self._dgraph = graph
        return self._dgraph

    def energy_of(self, params):
        """MaxCut energy for ``params = gamma[0..p) + beta[0..p)`` (host
        doubles) by one graph replay and one synchronisation."""
        if self._graph is None:
            self._capture()
            self._host_params_np = self.host_params.numpy()
            self._host_energy_np = self.host_energy.numpy()
            self._done = torch.cuda.Event()
        self._host_params_np[:] = params
        self._graph.replay()
        self._done.record(torch.cuda.current_stream(self.device))
        self._done.synchronize()
        return float(self._host_energy_np[0])


class QAOAEnergyEngine:
    """QAOA energy expectations contracted on the GPU.

    composer: ``'default'`` (ZZ gates + commutation simplifier, QTensor's
    ``DefaultQAOAComposer``), ``'zz'`` or ``'cx'``.
    ordering: ``'native'`` (C++ lightcones, multithreaded, and the cheapest of
    the reference greedy order, ``order_trials`` randomized greedy orders and
    minimum-fill orders per network) or ``'reference'`` (QTensor's exact
    qubit numbering and greedy elimination order).
    max_width / max_slices: a circuit whose width reaches ``max_width`` is
    sliced into at most ``max_slices`` networks (FeynmanSimulator's scheme,
    qtensor/FeynmanSimulator.py:49-84); the default 29 slices only what one
    B200's memory cannot hold unsliced.  slicing: ``'greedy'``
    (GreedyParvars), ``'tree_trim'`` (TreeTrimSplitter) or ``'late'``
    (LateParOptimizer) choice of the sliced variables.
    records: resolve every output element's operand offsets on the host, so
    that the shared-memory executor only loads and multiplies (same
    products, same order; off: the executor decodes the plan blobs).
    wave_ctas_per_sm: resident CTAs per SM of the wide networks' whole-GPU
    waves (0: as many as fit).
    dynamic_claims: persistent launches claim every network from their
    queue (for a GPU shared with other streams' kernels; off: each CTA starts
    on the job of its own index, which saves a queue round trip when the
    run has the GPU to itself).
    """

    def __init__(self, composer='default', ordering='native', device=None, threads=0,
                 cache_size=16, order_trials=16, autotune=True, max_width=29,
                 max_slices=1024, slicing='greedy', records=True, wave_ctas_per_sm=0,
                 dynamic_claims=False):
        _require_cuda()
        if ordering not in ('native', 'reference'):
            raise ValueError('ordering must be "native" or "reference"')
        self.composer = composer
        self.cid = composer_id(composer)
        self.ordering = ordering
        self.device = torch.device('cuda', torch.cuda.current_device() if device is None else device)
        self.threads = threads
        self.cache_size = cache_size
        self.order_trials = order_trials if ordering == 'native' else 0
        self.autotune = autotune
        self.max_width = max_width
        self.max_slices = max_slices
        self.slicing = slicing
        self.records = records
        self.wave_ctas_per_sm = wave_ctas_per_sm
        self.dynamic_claims = dynamic_claims
        self._cache = {}
        self._by_id = {}        # id(G) -> (weakref, nodes, p, key, edge count)
        self._edge_digests = {}  # id(edge subset) -> (subset, tuple, digest, length)
        self._lock = threading.Lock()
        _lib.check(_lib.lib().qtb_init(self.device.index))

    # ------------------------------------------------------------ compile
    def compile(self, G, p, gamma=None, beta=None, edges=None):
        """Compile (or fetch) the device plan of every edge of ``G`` at depth p
        (or of the edges whose indices in ``G.edges()`` order are ``edges``).

        The angles only steer the simplifier's near-zero cancellation test;
        a plan whose decisions depend on them is recompiled when they change."""
        return self._compile(G, p, self._params(p, gamma, beta), edges)

    def _compile(self, G, p, params, edges=None):
        """``compile`` with the angles already checked and packed."""
        key = self._key(G, p)
        if edges is not None:
            edges, digest = self._edges_digest(edges)
            key += ':' + digest
        with self._lock:
            cg = self._cache.get(key)
        if cg is not None and (not cg.angle_checks or cg.plan.params_valid(params)):
            return cg
        all_edges = list(G.edges())
        edges = all_edges if edges is None else [all_edges[i] for i in edges]
        if not edges:
            raise ValueError('no edges to compile')
        plan = NetworkPlan(2 * p)
        plan.set_order_trials(self.order_trials)
        plan.set_max_width(self.max_width, self.max_slices)
        plan.set_slicing(self.slicing)
        plan.set_records(self.records)
        plan.set_wave_ctas_per_sm(self.wave_ctas_per_sm)
        plan.set_dynamic_claims(self.dynamic_claims)
        if self.ordering == 'native':
            csr = graph_csr(G)
            index = {v: i for i, v in enumerate(csr[0])}
            pairs = np.array([(index[a], index[b]) for a, b in edges], dtype=np.int32)
            plan.add_lightcones(csr, pairs, p, self.cid, params, self.threads)
        else:
            passes = simplify_passes(self.cid)
            for edge in edges:
                nq, gates = reference_lightcone(G, edge, p, self.cid)
                plan.add_circuit(nq, gates, params, passes)
        plan.upload()
        plan.set_autotune(self.autotune)
        cg = CompiledGraph(plan, edges, p, self.composer, self.device)
        with self._lock:
            if len(self._cache) >= self.cache_size:
                self._cache.pop(next(iter(self._cache)))
            self._cache[key] = cg
        return cg

    def _key(self, G, p):
        """Plan-cache key of ``G``.  The full key hashes every edge; a graph
        object seen before with the same node count reuses its key without
        rehashing (networkx counts edges in O(nodes), which would cost more
        than a whole contraction), so call ``invalidate(G)`` after changing
        a graph's edges in place."""
        hit = self._by_id.get(id(G))
        if hit is not None:
            ref, n, hp, key, _ = hit
            if ref() is G and hp == p and n == len(G):
                return key
        key = graph_key(G, p, self.composer, self.ordering, self.order_trials,
                        (self.max_width, self.max_slices, self.slicing))
        try:
            self._by_id[id(G)] = (weakref.ref(G), len(G), p, key, G.number_of_edges())
        except TypeError:
            pass
        return key

    def _n_edges(self, G):
        """Edge count of ``G``, from the plan-cache entry of a graph object
        seen before (same rule as ``_key``), else counted."""
        hit = self._by_id.get(id(G))
        if hit is not None and hit[0]() is G and hit[1] == len(G):
            return hit[4]
        return G.number_of_edges()

    def _edges_digest(self, edges):
        """``(tuple of edge indices, digest)`` of an edge subset.  The digest
        of the last few subset tuples is kept (with a reference, so an id
        is not reused while it is cached): a caller that passes the same
        tuple every call, such as a rank's shard, pays for hashing once."""
        hit = self._edge_digests.get(id(edges))
        if hit is not None and hit[0] is edges and hit[3] == len(edges):
            return hit[1], hit[2]
        t = tuple(int(i) for i in edges)
        digest = hashlib.sha1(repr(t).encode()).hexdigest()
        if not isinstance(edges, tuple):      # a list may change in place: hash it every call
            return t, digest
        if len(self._edge_digests) >= 64:
            self._edge_digests.pop(next(iter(self._edge_digests)))
        self._edge_digests[id(edges)] = (edges, t, digest, len(edges))
        return t, digest

    def invalidate(self, G):
        """Forget cached plans of ``G`` (after changing it in place)."""
        hit = self._by_id.pop(id(G), None)
        if hit is not None:
            with self._lock:
                for k in [k for k in self._cache if k.split(':')[0] == hit[3]]:
                    self._cache.pop(k)

    @staticmethod
    def _params(p, gamma, beta):
        if gamma is None or beta is None:
            return np.zeros(2 * p)
        gamma = np.asarray(gamma, dtype=np.float64).ravel()
        beta = np.asarray(beta, dtype=np.float64).ravel()
        if len(gamma) != len(beta) or len(gamma) != p:
            raise ValueError('gamma and beta must both have length p={}'.format(p))
        return np.concatenate([gamma, beta])

    # ------------------------------------------------------------ run
    def energy_expectation(self, G, gamma, beta, path='batched', edges=None):
        """Expected MaxCut value of the depth-p QAOA state (p = len(gamma)).

        path: ``'batched'`` (whole-network executor, one graph replay) or
        ``'plain'`` (one bucket-kernel launch per bucket).  With ``edges``
        (indices into ``G.edges()``) the value is the share of those edges,
        ``(len(edges) - Re sum of their terms) / 2``: shares of disjoint edge
        sets add up to the energy."""
        gamma = np.asarray(gamma, dtype=np.float64).ravel()
        p = len(gamma)
        if (edges is not None and len(edges) == 0) or self._n_edges(G) == 0:
            self._params(p, gamma, beta)       # same argument checks
            return 0.0                         # an empty sum of edge terms (QAOASimulator.py:27-41)
        params = self._params(p, gamma, beta)
        cg = self._compile(G, p, params, edges)
        if path == 'batched':
            return cg.energy_of(params)
        self._launch(cg, p, gamma, beta, path)
        return float(cg.energy.cpu()[0])

    def edge_terms(self, G, gamma, beta, path='batched', edges=None):
        """``<Z_u Z_v>`` of every edge (numpy complex, edge order of ``G.edges()``,
        or of ``edges``; sliced edges are summed over their slices)."""
        gamma = np.asarray(gamma, dtype=np.float64).ravel()
        p = len(gamma)
        if (edges is not None and len(edges) == 0) or self._n_edges(G) == 0:
            self._params(p, gamma, beta)
            return np.zeros(0, dtype=np.complex128)
        cg = self.compile(G, p, gamma, beta, edges)
        self._launch(cg, p, gamma, beta, path)
        return cg.edge_terms()

    def _launch(self, cg, p, gamma, beta, path):
        if path not in ('batched', 'plain'):
            raise ValueError('path must be "batched" or "plain"')
        cg.params.copy_(torch.from_numpy(self._params(p, gamma, beta)))
        if path == 'batched':
            cg.launch()
        else:
            cg.launch_plain()

    def check_device(self, cg):
        """Raise if a kernel of ``cg`` reported an error status (synchronises)."""
        status = cg.plan.device_status()
        if status:
            raise _lib.QtbError(_lib.QTB_ERR_DEVICE, 'device status word {:#x}'.format(status))
