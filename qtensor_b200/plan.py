"""Compiled network plans: a thin owner of ``qtb_plan`` (``include/qtb.h``).

A plan holds any number of bucket networks (one per QAOA edge term, or one
per circuit), compiled on the host by the C++ plan compiler and contracted
on the device by ``qtb_plan_run``.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, ptr


def graph_csr(G):
    """``(nodes, indptr, indices)`` of a networkx graph; node ``nodes[i]`` is id ``i``."""
    nodes = list(G.nodes())
    index = {v: i for i, v in enumerate(nodes)}
    indptr = np.zeros(len(nodes) + 1, dtype=np.int64)
    indices = []
    for i, v in enumerate(nodes):
        nbrs = [index[w] for w in G[v] if w != v]
        indices.extend(nbrs)
        indptr[i + 1] = indptr[i] + len(nbrs)
    return nodes, indptr, np.asarray(indices, dtype=np.int32)


class NetworkPlan:
    """A set of compiled networks sharing ``n_params`` angle parameters."""

    def __init__(self, n_params):
        self._lib = _lib.lib()
        handle = ctypes.c_void_p()
        check(self._lib.qtb_plan_create(int(n_params), ctypes.byref(handle)))
        self._h = handle
        self.n_params = int(n_params)
        self.uploaded = False

    # ------------------------------------------------------------ compile
    def set_max_width(self, max_width, max_slices=256):
        """Slice circuits added afterwards whose greedy width reaches
        ``max_width`` into 2^k networks (0 = never); a circuit that would
        need more than ``max_slices`` networks fails to compile."""
        check(self._lib.qtb_plan_set_max_width(self._h, int(max_width), int(max_slices)))

    def set_slicing(self, method):
        """How circuits added afterwards choose sliced variables: ``'greedy'``
        (GreedyParvars, the default), ``'tree_trim'`` (TreeTrimSplitter) or
        ``'late'`` (LateParOptimizer)."""
        code = {'greedy': _lib.SLICE_GREEDY, 'tree_trim': _lib.SLICE_TREE_TRIM,
                'late': _lib.SLICE_LATE}[method]
        check(self._lib.qtb_plan_set_slicing(self._h, code))

    def groups(self):
        """Circuit (group) of every network."""
        return np.array([self.info(i)['group'] for i in range(len(self))], dtype=np.int64)

    def set_order_trials(self, trials):
        """Randomized greedy orders tried per network added afterwards (0 =
        the reference's greedy order only)."""
        check(self._lib.qtb_plan_set_order_trials(self._h, int(trials)))

    def set_share_lightcones(self, enable):
        """Compile edges with isomorphic lightcones once and copy the networks
        (default on; only ``add_lightcones`` made afterwards)."""
        check(self._lib.qtb_plan_set_share_lightcones(self._h, 1 if enable else 0))

    def set_records(self, enable):
        """Per-element operand records for the shared-memory executors
        (default on; set before ``upload``)."""
        check(self._lib.qtb_plan_set_records(self._h, 1 if enable else 0))

    def add_circuit(self, n_qubits, gates, params, simplify_passes=0):
        gates = np.ascontiguousarray(gates, dtype=_lib.GATE_DTYPE)
        params = np.ascontiguousarray(params, dtype=np.float64)
        idx = ctypes.c_int32()
        check(self._lib.qtb_plan_add_circuit(self._h, int(n_qubits), ptr(gates), len(gates),
                                             int(simplify_passes), ptr(params), ctypes.byref(idx)))
        self.uploaded = False
        return idx.value

    def add_circuit_batch(self, n_qubits, gates, params, batch_vars, simplify_passes=0):
        """Networks of the 2^batch_vars amplitudes <b|U|0> (b over qubits
        0..batch_vars-1, qubit 0 most significant); returns (first network,
        first group): amplitude i is group first_group + i."""
        gates = np.ascontiguousarray(gates, dtype=_lib.GATE_DTYPE)
        params = np.ascontiguousarray(params, dtype=np.float64)
        idx, grp = ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.qtb_plan_add_circuit_batch(self._h, int(n_qubits), ptr(gates), len(gates),
                                                   int(simplify_passes), ptr(params), int(batch_vars),
                                                   ctypes.byref(idx), ctypes.byref(grp)))
        self.uploaded = False
        return idx.value, grp.value

    def add_lightcones(self, csr, edges, p, composer, params, threads=0):
        """Compile the lightcone network of every edge (pairs of node ids)."""
        _, indptr, indices = csr
        edges = np.ascontiguousarray(edges, dtype=np.int32).reshape(-1, 2)
        params = np.ascontiguousarray(params, dtype=np.float64)
        first = ctypes.c_int32()
        check(self._lib.qtb_plan_add_lightcones(
            self._h, len(indptr) - 1, ptr(indptr), ptr(indices), ptr(edges), len(edges),
            int(p), int(composer), ptr(params), int(threads), ctypes.byref(first)))
        self.uploaded = False
        return first.value

    # ------------------------------------------------------------ queries
    def __len__(self):
        n = ctypes.c_int32()
        check(self._lib.qtb_plan_n_networks(self._h, ctypes.byref(n)))
        return n.value

    def info(self, i):
        info = _lib.NetworkInfo()
        check(self._lib.qtb_plan_network_info(self._h, int(i), ctypes.byref(info)))
        return info.as_dict()

    def infos(self):
        return [self.info(i) for i in range(len(self))]

    def peo(self, i):
        n = ctypes.c_int32()
        check(self._lib.qtb_plan_network_peo(self._h, int(i), None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=np.int32)
        check(self._lib.qtb_plan_network_peo(self._h, int(i), ptr(out), n.value, ctypes.byref(n)))
        return out.tolist()

    def params_valid(self, params):
        params = np.ascontiguousarray(params, dtype=np.float64)
        ok = ctypes.c_int32()
        check(self._lib.qtb_plan_check_params(self._h, ptr(params), ctypes.byref(ok)))
        return bool(ok.value)

    def export(self):
        """Host copies of the flattened plan arrays (numpy structured arrays)."""
        out = {}
        for which, (name, dtype) in enumerate([('nets', _lib.NET_DTYPE), ('ops', _lib.OP_DTYPE),
                                               ('ins', _lib.IN_DTYPE), ('phases', _lib.PHASE_DTYPE),
                                               ('entries', _lib.ENTRY_DTYPE),
                                               ('terms', _lib.TERM_DTYPE),
                                               ('runs', _lib.RUN_DTYPE),
                                               ('blobs', np.dtype('u1')),
                                               ('recs', np.dtype('<u4'))]):
            size = ctypes.c_size_t()
            check(self._lib.qtb_plan_export(self._h, which, None, 0, ctypes.byref(size)))
            buf = np.zeros(size.value // dtype.itemsize, dtype=dtype)
            check(self._lib.qtb_plan_export(self._h, which, ptr(buf), size.value, ctypes.byref(size)))
            out[name] = buf
        n = ctypes.c_int64()
        check(self._lib.qtb_plan_table_elems(self._h, ctypes.byref(n)))
        out['table_elems'] = n.value
        return out

    # ------------------------------------------------------------ device
    def upload(self):
        check(self._lib.qtb_plan_upload(self._h))
        self.uploaded = True

    def scratch_bytes(self, first=0, count=None):
        count = len(self) - first if count is None else count
        n = ctypes.c_size_t()
        check(self._lib.qtb_plan_scratch_bytes(self._h, int(first), int(count), ctypes.byref(n)))
        return n.value

    def run(self, first, count, params_dev, terms_dev, energy_dev=None, scratch_dev=None,
            stream=0):
        """Asynchronous contraction of networks [first, first+count) on ``stream``."""
        check(self._lib.qtb_plan_run(self._h, int(first), int(count), ptr(params_dev),
                                     ptr(terms_dev), ptr(energy_dev), ptr(scratch_dev),
                                     ctypes.c_void_p(int(stream))))

    def plain_scratch_bytes(self, first=0, count=None):
        count = len(self) - first if count is None else count
        n = ctypes.c_size_t()
        check(self._lib.qtb_plan_plain_scratch_bytes(self._h, int(first), int(count),
                                                     ctypes.byref(n)))
        return n.value

    def run_plain(self, first, count, params_dev, terms_dev, energy_dev=None, scratch_dev=None,
                  stream=0):
        """The plain path: one bucket kernel launch per bucket of networks
        [first, first+count), intermediates in ``scratch_dev`` (global
        memory of ``plain_scratch_bytes``), asynchronous on ``stream``."""
        nbytes = 0 if scratch_dev is None else scratch_dev.numel() * scratch_dev.element_size()
        check(self._lib.qtb_plan_run_plain(self._h, int(first), int(count), ptr(params_dev),
                                           ptr(terms_dev), ptr(energy_dev), ptr(scratch_dev),
                                           nbytes, ctypes.c_void_p(int(stream))))

    def set_wave_ctas_per_sm(self, ctas):
        """Resident CTAs per SM of the wide waves (0: as many as fit); set
        before the first run."""
        check(self._lib.qtb_plan_set_wave_ctas_per_sm(self._h, int(ctas)))

    def set_dynamic_claims(self, enable):
        """Persistent launches claim every network from their queue (for a
        GPU shared with other streams' kernels) instead of starting each CTA
        on the job of its own index; results are the same."""
        check(self._lib.qtb_plan_set_dynamic_claims(self._h, int(bool(enable))))

    def set_autotune(self, enable):
        """Time every launch class with 64..1024 threads per CTA on the first
        run of a range and keep the fastest."""
        check(self._lib.qtb_plan_set_autotune(self._h, 1 if enable else 0))

    def last_launch_config(self):
        """[(networks, threads, smem bytes, flags)] of the latest run's
        schedule; flags: 1 shared-memory arena, 2 persistent launch."""
        n = ctypes.c_int32()
        out = np.zeros(4 * 16, dtype=np.int32)
        check(self._lib.qtb_plan_last_launch_config(self._h, ptr(out), len(out), ctypes.byref(n)))
        return [tuple(int(x) for x in out[4 * c:4 * c + 4]) for c in range(min(n.value, 16))]

    def device_bytes(self):
        """Device memory the uploaded plan holds (excluding run buffers)."""
        n = ctypes.c_size_t()
        check(self._lib.qtb_plan_device_bytes(self._h, ctypes.byref(n)))
        return n.value

    def device_status(self):
        s = ctypes.c_int32()
        check(self._lib.qtb_plan_device_status(self._h, ctypes.byref(s)))
        return s.value

    def set_timing(self, enable):
        check(self._lib.qtb_plan_set_timing(self._h, 1 if enable else 0))

    def collect_timing(self):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        check(self._lib.qtb_plan_collect_timing(self._h, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def close(self):
        if getattr(self, '_h', None):
            self._lib.qtb_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
