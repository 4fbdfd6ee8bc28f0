"""Generate the golden amplitude-batch fixtures from the reference QTensor code.

Runs the reference's own ``QtreeSimulator.simulate_batch`` (qtensor/Simulate.py:66-94,
imported from a read-only reference checkout through ``oracle/refimport.py``,
on the oracle ``qtree``) on seeded random circuits and writes
``batch_reference.json`` next to this script: every circuit as a list of
``[name, qubits, alpha]`` (alpha null for fixed gates, '+' marking a dagger)
with the amplitudes for several ``batch_vars``.  The GPU box has no reference
checkout; the tests read only the JSON.

    python tests/golden/make_batch_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))

from refimport import import_reference  # noqa: E402


def random_circuit(rng, n_qubits, n_layers, ops, zz):
    """Layers of one-qubit gates and entanglers on random pairs; about a
    quarter of the gates daggered."""
    circuit = [ops.H(q) for q in range(n_qubits)]
    one = [ops.X, ops.Y, ops.Z, ops.T, ops.H]
    rot = [ops.ZPhase, ops.XPhase, ops.YPhase]
    for _ in range(n_layers):
        for q in range(n_qubits):
            if rng.random() < 0.5:
                g = rot[rng.integers(len(rot))](q, alpha=float(rng.uniform(-1, 1)))
            else:
                g = one[rng.integers(len(one))](q)
            if rng.random() < 0.25:
                g.dagger_me()
            circuit.append(g)
        a, b = (int(x) for x in rng.choice(n_qubits, size=2, replace=False))
        kind = rng.integers(3)
        if kind == 0:
            circuit.append(ops.cX(a, b))
        elif kind == 1:
            circuit.append(ops.cZ(a, b))
        else:
            g = zz(a, b, alpha=float(rng.uniform(-1, 1)))
            if rng.random() < 0.25:
                g.dagger_me()
            circuit.append(g)
    return circuit


def encode(circuit):
    out = []
    for g in circuit:
        alpha = g.parameters.get('alpha') if g.parameters else None
        out.append([g.name, [int(q) for q in g.qubits], None if alpha is None else float(alpha)])
    return out


def main():
    qtensor = import_reference()
    if qtensor is None:
        sys.exit('no reference checkout found (set QTENSOR_REFERENCE)')
    import qtree.operators as ops
    from qtensor.OpFactory import ZZ
    from qtensor.Simulate import QtreeSimulator

    rng = np.random.default_rng(7)
    cases = []
    for n_qubits, n_layers, batches in [(4, 6, [0, 1, 2, 4]), (6, 8, [0, 3]), (8, 10, [0, 2, 5]),
                                        (10, 6, [0, 4])]:
        circuit = random_circuit(rng, n_qubits, n_layers, ops, ZZ)
        entry = {'n_qubits': n_qubits, 'gates': encode(circuit), 'amplitudes': {}}
        for k in batches:
            amps = QtreeSimulator().simulate_batch(circuit, batch_vars=k)
            entry['amplitudes'][str(k)] = [[float(z.real), float(z.imag)] for z in np.ravel(amps)]
        cases.append(entry)
        print('circuit n={} gates={} batches={}'.format(n_qubits, len(circuit), batches), flush=True)
    with open(os.path.join(HERE, 'batch_reference.json'), 'w') as f:
        json.dump({'generator': 'tests/golden/make_batch_golden.py', 'cases': cases}, f,
                  separators=(',', ':'))


if __name__ == '__main__':
    main()
