"""Amplitude simulation of arbitrary circuits on one B200.

``QtreeSimulator`` mirrors the reference's ``QtreeSimulator``
(qtensor/Simulate.py:22-94): ``simulate_batch(qc, batch_vars)`` returns the
2^batch_vars amplitudes ``<b 0..0| U |0..0>`` over the first ``batch_vars``
qubits, flattened with qubit 0 as the most significant bit, like the
reference's output tensor over its free variables; ``simulate`` and
``simulate_state`` are ``batch_vars=0``.  The contraction runs through the
same plan compiler and device executor as the QAOA engine: every output
bitstring is one network with its bra values fixed (plus its slices when
the width reaches ``max_width``), all contracted in one launch.

Circuits are lists of the reference's qtree gate objects -- anything with
``name``, ``qubits`` and (for rotations) ``parameters['alpha']`` -- or a
``qtensor_b200._lib.GATE_DTYPE`` array with its parameter vector.
Supported gates: M, I, H, X, Y, Z, T, cX, cZ, ZPhase, XPhase, YPhase, ZZ and
their daggers (name suffix '+': rotations with the angle negated, T+ as
ZPhase(-1/4), the others self-adjoint).
"""
import numpy as np
import torch

from . import _lib
from .plan import NetworkPlan

_FIXED = {'M': _lib.GATE_M, 'H': _lib.GATE_H, 'X': _lib.GATE_X, 'Y': _lib.GATE_Y,
          'Z': _lib.GATE_Z, 'T': _lib.GATE_T, 'cX': _lib.GATE_CX, 'cZ': _lib.GATE_CZ}
_ROTATIONS = {'ZPhase': _lib.GATE_ZPHASE, 'XPhase': _lib.GATE_XPHASE,
              'YPhase': _lib.GATE_YPHASE, 'ZZ': _lib.GATE_ZZ}


def _attr(gate, name):
    v = getattr(gate, name)
    return v() if callable(v) else v


def gates_from_circuit(qc):
    """(n_qubits, gate array, params) of a list of qtree-style gate objects:
    every rotation angle becomes its own parameter (coefficient 1)."""
    rows, params, n_qubits = [], [], 0
    for gate in qc:
        name = str(_attr(gate, 'name'))
        dagger = name.endswith('+')
        base = name.rstrip('+')
        qubits = [int(q) for q in _attr(gate, 'qubits')]
        if qubits:
            n_qubits = max(n_qubits, max(qubits) + 1)
        if base == 'I':
            continue
        q0 = qubits[0]
        q1 = qubits[1] if len(qubits) > 1 else -1
        if base in _FIXED:
            if base == 'T' and dagger:
                params.append(-0.25)
                rows.append((_lib.GATE_ZPHASE, q0, -1, len(params) - 1, 1.0))
            else:
                rows.append((_FIXED[base], q0, q1, -1, 0.0))
        elif base in _ROTATIONS:
            alpha = float(_attr(gate, 'parameters')['alpha'])
            params.append(-alpha if dagger else alpha)
            rows.append((_ROTATIONS[base], q0, q1, len(params) - 1, 1.0))
        else:
            raise NotImplementedError('gate {!r} is not supported'.format(name))
    return n_qubits, np.array(rows, dtype=_lib.GATE_DTYPE), np.array(params, dtype=np.float64)


class QtreeSimulator:
    """``simulate_batch`` / ``simulate`` / ``simulate_state`` of the reference
    simulator, contracted on the GPU (complex64 products, amplitudes summed
    over slices in fp64 on the host).

    max_tw: like the reference, a ``ValueError`` when the contraction width
    exceeds it (before slicing); max_width / max_slices: circuits whose width
    reaches max_width are sliced into at most max_slices networks per
    amplitude; slicing: how the sliced variables are chosen (``'greedy'``,
    ``'tree_trim'`` or ``'late'``, see ``NetworkPlan.set_slicing``);
    order_trials: extra randomized greedy orders per network."""

    def __init__(self, device=None, max_tw=None, max_width=26, max_slices=256, order_trials=8,
                 slicing='greedy'):
        if not torch.cuda.is_available():
            raise RuntimeError('qtensor_b200 needs a CUDA device; there is no CPU fallback')
        self.device = torch.device('cuda', torch.cuda.current_device() if device is None else device)
        self.max_tw = max_tw
        self.max_width = max_width
        self.max_slices = max_slices
        self.order_trials = order_trials
        self.slicing = slicing
        _lib.check(_lib.lib().qtb_init(self.device.index))
        self.plan = None

    def _compile(self, qc, batch_vars, params=None):
        if isinstance(qc, np.ndarray):
            gates = np.ascontiguousarray(qc, dtype=_lib.GATE_DTYPE)
            params = np.zeros(0) if params is None else np.asarray(params, dtype=np.float64)
            used = [int(g['q0']) for g in gates] + [int(g['q1']) for g in gates if g['q1'] >= 0]
            n_qubits = max(used) + 1 if used else 0
        else:
            n_qubits, gates, params = gates_from_circuit(qc)
        n_qubits = max(n_qubits, batch_vars, 1)
        plan = NetworkPlan(len(params))
        plan.set_order_trials(self.order_trials)
        plan.set_max_width(self.max_width, self.max_slices)
        plan.set_slicing(self.slicing)
        first, group0 = plan.add_circuit_batch(n_qubits, gates, params, batch_vars)
        if self.max_tw is not None:
            width = max(i['treewidth'] for i in plan.infos())
            if width > self.max_tw:
                plan.close()
                raise ValueError('Treewidth {} is larger than max_tw={}.'.format(width, self.max_tw))
        return plan, params, group0

    def simulate_batch(self, qc, batch_vars=0, peo=None, params=None):
        """Amplitudes of the 2^batch_vars output bitstrings of qubits
        0..batch_vars-1 (others 0), qubit 0 the most significant bit."""
        if peo is not None:
            raise NotImplementedError('a given elimination order is not supported; '
                                      'the plan compiler chooses its own')
        plan, params, group0 = self._compile(qc, int(batch_vars), params)
        try:
            with torch.cuda.device(self.device):
                plan.upload()
                n = len(plan)
                params_dev = torch.from_numpy(params).to(self.device) if len(params) else None
                terms = torch.empty(n, dtype=torch.complex64, device=self.device)
                nbytes = plan.scratch_bytes(0, n)
                scratch = torch.empty(nbytes, dtype=torch.uint8, device=self.device) if nbytes else None
                stream = torch.cuda.current_stream(self.device)
                plan.run(0, n, params_dev, terms, None, scratch, stream.cuda_stream)
                vals = terms.cpu().numpy().astype(np.complex128)
                status = plan.device_status()
                if status:
                    raise _lib.QtbError(_lib.QTB_ERR_DEVICE, 'device status word {:#x}'.format(status))
            out = np.zeros(1 << int(batch_vars), dtype=np.complex128)
            np.add.at(out, plan.groups() - group0, vals)
            return out
        finally:
            plan.close()

    def simulate(self, qc):
        return self.simulate_state(qc)

    def simulate_state(self, qc, peo=None):
        return self.simulate_batch(qc, batch_vars=0, peo=peo)


class SlicesOptimizer:
    """Choice of parallel (sliced) variables of ``FeynmanSimulator``
    (qtensor/optimisation/Optimizer.py:90-159): variables of highest degree
    (GreedyParvars) until the width drops below ``max_tw - tw_bias``.  Only
    the slicing parameters are kept: the plan compiler does the work."""
    method = 'greedy'

    def __init__(self, tw_bias=2, max_tw=None, **kwargs):
        self.tw_bias = tw_bias
        self.max_tw = kwargs.get('target_tw') or max_tw

    def max_width(self, default_max_tw):
        """The plan compiler's ``max_width``: slice while width >= it."""
        max_tw = default_max_tw if self.max_tw is None else self.max_tw
        return max(1, int(max_tw) - int(self.tw_bias))


class TreeTrimSplitter(SlicesOptimizer):
    """TreeTrimSplitter (qtensor/optimisation/Optimizer.py:178-224): rounds of
    int(0.2 x excess) + 1 variables from the largest elimination cliques,
    until the width is at most ``max_tw - tw_bias``."""
    method = 'tree_trim'

    def max_width(self, default_max_tw):
        return super().max_width(default_max_tw) + 1


class LateParOptimizer:
    """LateParOptimizer (qtensor/optimisation/late_parallelisation.py:30-202)
    with one variable per bunch: each variable is sliced at the step of the
    elimination order that leaves the least width, until the width is at
    most ``target_tw``."""
    method = 'late'

    def __init__(self, target_tw=None, par_vars=None, p_bunch=None, n_bunches=None,
                 ordering_algo='greedy', slicing_algo='greedy'):
        if ordering_algo != 'greedy' or slicing_algo != 'greedy':
            raise ValueError('only the greedy ordering and slicing algorithms are supported')
        if par_vars is not None or n_bunches is not None:
            raise NotImplementedError('a fixed number of sliced variables is not supported; give target_tw')
        self.target_tw = target_tw

    def max_width(self, default_max_tw):
        target = default_max_tw if self.target_tw is None else self.target_tw
        return max(1, int(target) + 1)


class FeynmanSimulator(QtreeSimulator):
    """``FeynmanSimulator.simulate`` / ``simulate_batch_adaptive``
    (qtensor/FeynmanSimulator.py:27-100): the circuit is sliced over parallel
    variables, chosen greedily by degree until its width drops below
    ``max_tw - tw_bias`` (``SlicesOptimizer``, qtensor/optimisation/
    Optimizer.py:88-160), and the amplitudes of all 2^k paths are summed.
    Assigning ``sim.optimizer = TreeTrimSplitter(...)`` or
    ``LateParOptimizer(target_tw=...)`` selects those choices instead, as
    the reference's tests do (qtensor/tests/test_qaoa_energy.py:116-117).
    Here every path is one network of a single launch, so ``pool_type`` and
    ``n_processes`` have nothing to do.  ``max_tw`` defaults, like the
    reference's memory rule, to log2 of the device's free bytes over the
    8-byte complex64 element.  At most ``max_slices`` paths per amplitude."""

    def __init__(self, *args, pool_type='process', n_processes=None, max_tw=None, max_slices=4096,
                 **kwargs):
        super().__init__(*args, max_slices=max_slices, **kwargs)
        self.slice_max_tw = max_tw
        self.optimizer = None
        self.pool_type = pool_type
        self.n_processes = 2 if n_processes is None else n_processes

    def _target_width(self, tw_bias):
        max_tw = self.slice_max_tw
        if max_tw is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            max_tw = int(np.log2(free)) - 3
        return max(1, int(max_tw) - int(tw_bias))

    def simulate(self, qc, batch_vars=0, tw_bias=2):
        return self.simulate_batch_adaptive(qc, batch_vars, tw_bias=tw_bias)

    def simulate_batch_adaptive(self, qc, batch_vars=0, tw_bias=2):
        if self.optimizer is None:
            self.max_width = self._target_width(tw_bias)
            self.slicing = 'greedy'
        else:
            self.max_width = self.optimizer.max_width(self._target_width(0))
            self.slicing = self.optimizer.method
        return self.simulate_batch(qc, batch_vars=batch_vars)
