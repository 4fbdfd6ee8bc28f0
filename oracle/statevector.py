"""Independent physics oracles for QAOA MaxCut energies.

TEST INFRASTRUCTURE ONLY.  These do not follow the reference's tensor-network
algorithm at all; they pin ``oracle/qtree`` + ``oracle/qtensor_port.py``
physically:

* ``qaoa_energy_statevector`` -- dense state vector, N <= ~22 qubits;
* ``qaoa_p1_edge_term`` -- closed-form p=1 edge expectation for arbitrary
  graphs (Wang, Hadfield, Jiang, Rieffel, Phys. Rev. A 97, 022304 (2018),
  Theorem 1).

Angle convention of QTensor (``qtensor/CircuitComposer.py:109-111,168-169``):
the cost layer is ``prod_edges ZZ(alpha=2*gamma) = exp(-i pi gamma Z_u Z_v)``
and the mixer ``XPhase(alpha=2*beta) ~ exp(-i pi beta X)``; the energy is the
expected cut ``sum_edges (1 - <Z_u Z_v>) / 2`` (``qtensor/QAOASimulator.py:27-41``).
"""
import numpy as np


def _cut_diagonal(G, nodes):
    """Per basis state: sum over edges of z_u z_v (z = +-1), qubit k = bit k
    (most significant first) of the state index."""
    n = len(nodes)
    pos = {v: k for k, v in enumerate(nodes)}
    idx = np.arange(2 ** n, dtype=np.int64)
    z = 1 - 2 * ((idx[None, :] >> (n - 1 - np.arange(n)[:, None])) & 1)
    zz = {}
    for u, v in G.edges():
        zz[(u, v)] = z[pos[u]] * z[pos[v]]
    return zz


def qaoa_edge_terms_statevector(G, gamma, beta):
    """``{edge: <Z_u Z_v>}`` after the depth-p QAOA state on all of ``G``."""
    nodes = list(G.nodes())
    n = len(nodes)
    if n > 24:
        raise ValueError('state vector oracle is limited to 24 qubits')
    zz = _cut_diagonal(G, nodes)
    total_zz = sum(zz.values()) if zz else np.zeros(2 ** n)
    psi = np.full(2 ** n, 2.0 ** (-n / 2), dtype=np.complex128)
    for g, b in zip(gamma, beta):
        psi = psi * np.exp(-1j * np.pi * g * total_zz)
        c, s = np.cos(np.pi * b), np.sin(np.pi * b)
        for k in range(n):
            t = psi.reshape(2 ** k, 2, 2 ** (n - k - 1))
            a0, a1 = t[:, 0, :].copy(), t[:, 1, :].copy()
            t[:, 0, :] = c * a0 - 1j * s * a1
            t[:, 1, :] = -1j * s * a0 + c * a1
    prob = np.abs(psi) ** 2
    return {e: float(np.dot(prob, d)) for e, d in zz.items()}


def qaoa_energy_statevector(G, gamma, beta):
    terms = qaoa_edge_terms_statevector(G, gamma, beta)
    return (G.number_of_edges() - sum(terms.values())) / 2


def qaoa_p1_edge_term(G, edge, gamma, beta):
    """Closed-form ``<Z_u Z_v>`` for p=1 in QTensor's angle convention."""
    u, v = edge
    g = -2 * np.pi * gamma          # QTensor gamma -> exp(-i g C), C = sum (1 - ZZ)/2
    b = np.pi * beta                # QTensor beta  -> exp(-i b sum X)
    du = G.degree(u) - 1
    dv = G.degree(v) - 1
    lam = len(set(G[u]) & set(G[v]) - {u, v})
    c_uv = (0.5 + 0.25 * np.sin(4 * b) * np.sin(g) * (np.cos(g) ** du + np.cos(g) ** dv)
            - 0.25 * np.sin(2 * b) ** 2 * np.cos(g) ** (du + dv - 2 * lam)
            * (1 - np.cos(2 * g) ** lam))
    return 1 - 2 * c_uv


def _gate_matrix(name, alpha):
    """Standard matrix of a gate (qubit order of its arguments, first
    argument most significant); '+' suffix: conjugate transpose."""
    dagger = name.endswith('+')
    base = name.rstrip('+')
    r2 = 1 / np.sqrt(2)
    if base == 'H':
        m = np.array([[r2, r2], [r2, -r2]])
    elif base == 'X':
        m = np.array([[0, 1], [1, 0]], dtype=complex)
    elif base == 'Y':
        m = np.array([[0, -1j], [1j, 0]])
    elif base == 'Z':
        m = np.diag([1, -1]).astype(complex)
    elif base == 'T':
        m = np.diag([1, np.exp(1j * np.pi / 4)])
    elif base == 'cX':
        m = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=complex)
    elif base == 'cZ':
        m = np.diag([1, 1, 1, -1]).astype(complex)
    elif base == 'ZPhase':
        m = np.diag([1, np.exp(1j * np.pi * alpha)])
    elif base in ('XPhase', 'YPhase'):
        c, s = np.cos(np.pi * alpha / 2), np.sin(np.pi * alpha / 2)
        rot = (np.array([[c, -1j * s], [-1j * s, c]]) if base == 'XPhase'
               else np.array([[c, -s], [s, c]], dtype=complex))
        m = np.exp(1j * np.pi * alpha / 2) * rot
    elif base == 'ZZ':
        p = np.exp(1j * np.pi * alpha / 2)
        m = np.diag([1 / p, p, p, 1 / p])
    else:
        raise ValueError(name)
    return m.conj().T if dagger else m


def circuit_state(gates, n_qubits):
    """Dense ``U |0...0>`` of ``gates`` = [(name, qubits, alpha), ...],
    applied in list order; qubit 0 is the most significant bit."""
    psi = np.zeros(2 ** n_qubits, dtype=complex)
    psi[0] = 1
    psi = psi.reshape([2] * n_qubits)
    for name, qubits, alpha in gates:
        m = _gate_matrix(name, alpha)
        k = len(qubits)
        m = m.reshape([2] * (2 * k))
        psi = np.tensordot(m, psi, axes=(list(range(k, 2 * k)), list(qubits)))
        psi = np.moveaxis(psi, list(range(k)), list(qubits))
    return psi.reshape(-1)
