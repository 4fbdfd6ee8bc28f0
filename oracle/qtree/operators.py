"""Gate classes with their tensors in qtree's compact layout.

Oracle restatement (test infrastructure only).  Conventions, pinned by
``qtensor/tests/test_qaoa_energy.py:58`` + ``qtensor/tests/qiskit_qaoa_energy.py:107``
(ZZ(2*gamma) == rzz(2*pi*gamma), XPhase(2*beta) == rx(2*pi*beta) up to phase)
and by ``qtensor/OpFactory.py:17-27`` (cirq ``ZPowGate``/``XPowGate`` exponent
``alpha``):

* a gate lists in ``_changes_qubits`` the positions of the qubits that get a
  new variable; diagonal action on a qubit uses a single index, so ``Z``,
  ``ZPhase``, ``cZ`` and ``ZZ`` tensors are vectors / 2x2 arrays over existing
  variables and ``cX`` is ``[control][target_out][target_in]``;
* ``ZPhase(alpha) = diag(1, e^{i pi alpha})``;
  ``XPhase(alpha) = e^{i pi alpha/2} (cos(pi alpha/2) I - i sin(pi alpha/2) X)``;
  ``YPhase(alpha) = e^{i pi alpha/2} (cos(pi alpha/2) I - i sin(pi alpha/2) Y)``;
* ``dagger_me()`` keeps the class, appends ``'+'`` to ``name`` and keeps the
  original ``alpha`` (``qtensor/simplify_circuit/simplify_circuit_api.py:87-90``);
  the daggered tensor is the conjugate transpose of the original array
  (``qtensor/OpFactory.py:157-158`` builds inverses this way).
"""
import numpy as np


class Gate:
    """Base gate: ``qubits``, ``parameters`` (a dict; raises ``KeyError`` for
    missing entries), ``changed_qubits``, ``gen_tensor()`` and ``dagger_me()``."""
    _changes_qubits = ()

    def __init__(self, *qubits):
        if len(qubits) == 0:
            raise ValueError('{} needs at least one qubit'.format(type(self).__name__))
        self._qubits = tuple(int(q) for q in qubits)
        self._parameters = {}
        self._dagger = False
        # a subclass may fix its label with a class attribute ``name``
        # (``qtensor/OpFactory.py:32,45``); otherwise the class name is used
        self.name = next((k.__dict__['name'] for k in type(self).__mro__
                          if isinstance(k.__dict__.get('name'), str)),
                         type(self).__name__)

    @property
    def qubits(self):
        return self._qubits

    @property
    def parameters(self):
        return self._parameters

    @property
    def changed_qubits(self):
        return tuple(self._qubits[i] for i in self._changes_qubits)

    @property
    def is_dagger(self):
        return self._dagger

    def gen_tensor(self):
        raise NotImplementedError

    def dagger_me(self):
        self._dagger = not self._dagger
        self.name = self.name + '+' if self._dagger else self.name.rstrip('+')
        return self

    def __str__(self):
        params = ''
        if self._parameters:
            params = '[' + ','.join('{}={:.4f}'.format(k, v)
                                    for k, v in sorted(self._parameters.items())) + ']'
        return '{}{}({})'.format(self.name, params, ','.join(map(str, self._qubits)))

    __repr__ = __str__


class ParametricGate(Gate):
    parameter_count = 1

    def __init__(self, *qubits, **parameters):
        super().__init__(*qubits)
        self._parameters = dict(parameters)


def gate_tensor(op):
    """Array of ``op`` in its index layout, conjugate-transposed when daggered."""
    t = np.asarray(op.gen_tensor())
    if getattr(op, '_dagger', False):
        t = t.conj().T
    return t


class M(Gate):
    """Measurement / boundary tensor: identity between the frame var and a new var."""
    _changes_qubits = (0,)

    def gen_tensor(self):
        return np.eye(2, dtype=np.complex128)


class I(Gate):
    _changes_qubits = ()

    def gen_tensor(self):
        return np.ones(2, dtype=np.complex128)


class H(Gate):
    _changes_qubits = (0,)

    def gen_tensor(self):
        return np.array([[1, 1], [1, -1]], dtype=np.complex128) / np.sqrt(2)


class X(Gate):
    _changes_qubits = (0,)

    def gen_tensor(self):
        return np.array([[0, 1], [1, 0]], dtype=np.complex128)


class Y(Gate):
    _changes_qubits = (0,)

    def gen_tensor(self):
        return np.array([[0, -1j], [1j, 0]], dtype=np.complex128)


class Z(Gate):
    _changes_qubits = ()

    def gen_tensor(self):
        return np.array([1, -1], dtype=np.complex128)


class T(Gate):
    _changes_qubits = ()

    def gen_tensor(self):
        return np.array([1, np.exp(1j * np.pi / 4)], dtype=np.complex128)


class cX(Gate):
    """CNOT: diagonal on the control, ``[control][target_out][target_in]``."""
    _changes_qubits = (1,)

    def gen_tensor(self):
        t = np.zeros((2, 2, 2), dtype=np.complex128)
        t[0] = np.eye(2)
        t[1] = np.array([[0, 1], [1, 0]])
        return t


class cZ(Gate):
    _changes_qubits = ()

    def gen_tensor(self):
        return np.array([[1, 1], [1, -1]], dtype=np.complex128)


class ZPhase(ParametricGate):
    _changes_qubits = ()

    def gen_tensor(self):
        alpha = self._parameters['alpha']
        return np.array([1, np.exp(1j * np.pi * alpha)], dtype=np.complex128)


class XPhase(ParametricGate):
    _changes_qubits = (0,)

    def gen_tensor(self):
        alpha = self._parameters['alpha']
        c, s = np.cos(np.pi * alpha / 2), np.sin(np.pi * alpha / 2)
        g = np.exp(1j * np.pi * alpha / 2)
        return g * np.array([[c, -1j * s], [-1j * s, c]], dtype=np.complex128)


class YPhase(ParametricGate):
    _changes_qubits = (0,)

    def gen_tensor(self):
        alpha = self._parameters['alpha']
        c, s = np.cos(np.pi * alpha / 2), np.sin(np.pi * alpha / 2)
        g = np.exp(1j * np.pi * alpha / 2)
        return g * np.array([[c, -s], [s, c]], dtype=np.complex128)


LABEL_TO_GATE_DICT = {
    'i': I, 'h': H, 'x': X, 'y': Y, 'z': Z, 't': T,
    'cx': cX, 'cz': cZ,
    'rz': ZPhase, 'rx': XPhase, 'ry': YPhase,
}


def read_circuit_file(filename, max_depth=None):
    raise NotImplementedError('qsim circuit files are not part of the oracle')


def from_qiskit_circuit(qiskit_circ):
    raise NotImplementedError('qiskit is not installed')
