"""Import the reference ``qtensor`` package on top of the oracle ``qtree``.

TEST INFRASTRUCTURE ONLY, and only where a read-only checkout of the
reference exists (``QTENSOR_REFERENCE``, else a directory ``reference`` beside
this repository's root); the
fixture generator ``tests/golden/make_golden.py`` and the CPU test that pins
``oracle/qtensor_port.py`` against the reference use it.

The reference imports ``cirq`` (``qtensor/OpFactory.py:1``), ``pyrofiler``
(``qtensor/ProcessingFrameworks.py:8``) and ``matplotlib`` (``qtensor/utils.py:7``)
at import time; none is installed, and none is on the bucket-elimination
path, so minimal stand-ins are registered before the import.
"""
import contextlib
import os
import sys
import time
import types

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
# a checkout named ``reference`` next to the repository root
DEFAULT_REFERENCE = os.path.join(os.path.dirname(os.path.dirname(ORACLE_DIR)), 'reference')


def reference_root():
    root = os.environ.get('QTENSOR_REFERENCE', DEFAULT_REFERENCE)
    return root if os.path.isdir(os.path.join(root, 'qtensor')) else None


def _stub_modules():
    if 'cirq' not in sys.modules:
        cirq = types.ModuleType('cirq')
        for name in ('H', 'CX', 'Z', 'X', 'CZ'):
            setattr(cirq, name, object())

        class _Pow:
            def __init__(self, exponent=1.0):
                self.exponent = exponent

            def on(self, *qubits):
                raise NotImplementedError('cirq is not installed')
        cirq.ZPowGate = cirq.XPowGate = _Pow

        def _missing(*a, **k):
            raise NotImplementedError('cirq is not installed')
        cirq.LineQubit = cirq.Circuit = cirq.Simulator = cirq.inverse = _missing
        sys.modules['cirq'] = cirq

    if 'pyrofiler' not in sys.modules:
        prof = types.ModuleType('pyrofiler')

        @contextlib.contextmanager
        def timing(*args, callback=None, **kwargs):
            start = time.perf_counter()
            yield
            if callback is not None:
                callback(time.perf_counter() - start, *args)
        prof.timing = timing
        sys.modules['pyrofiler'] = prof

    if 'matplotlib' not in sys.modules:
        mpl = types.ModuleType('matplotlib')
        plt = types.ModuleType('matplotlib.pyplot')
        mpl.pyplot = plt
        sys.modules['matplotlib'] = mpl
        sys.modules['matplotlib.pyplot'] = plt


def import_reference():
    """Return the reference ``qtensor`` module, or ``None`` if no checkout exists."""
    root = reference_root()
    if root is None:
        return None
    if ORACLE_DIR not in sys.path:
        sys.path.insert(0, ORACLE_DIR)
    _stub_modules()
    if root not in sys.path:
        sys.path.append(root)
    import qtensor  # noqa: E402
    return qtensor
