"""``QAOASimulator`` under the reference's names (qtensor/QAOASimulator.py:12-108).

A user of ``QAOAQtreeSimulator(composer).energy_expectation(G, gamma, beta)``
switches by constructing ``QAOAQtreeSimulator(composer)`` from here: the
composer may be the reference's class (``DefaultQAOAComposer``,
``ZZQtreeQAOAComposer``, ``QtreeQAOAComposer``, matched by name) or
``'default'`` / ``'zz'`` / ``'cx'``.  ``energy_expectation_parallel`` runs the
same batched GPU contraction (process counts do not apply);
``energy_expectation_mpi`` shards the edges over an initialised
``torch.distributed`` group when there is one (every rank receives the
energy), and otherwise runs on this GPU.

The energies come back in the reference's shape: its per-edge amplitudes are
the flattened one-element arrays of ``QtreeSimulator.simulate`` and their sum
goes through ``_post_process_energy`` (qtensor/QAOASimulator.py:27-41), so a
graph with edges gives a float64 array of shape (1,) (callers index
``E[0]``), and a graph without edges the plain float 0.0.
"""
import numpy as np

from .engine import QAOAEnergyEngine

_COMPOSERS = {'DefaultQAOAComposer': 'default', 'ZZQtreeQAOAComposer': 'zz',
              'QtreeQAOAComposer': 'cx', 'default': 'default', 'zz': 'zz', 'cx': 'cx'}


def composer_name(composer):
    key = composer if isinstance(composer, str) else getattr(composer, '__name__', type(composer).__name__)
    if key not in _COMPOSERS:
        raise ValueError('composer {!r} is not supported'.format(key))
    return _COMPOSERS[key]


def _reference_shape(G, E):
    """``_post_process_energy``'s result type for an energy ``E``."""
    if G.number_of_edges() == 0:
        return 0.0
    return np.array([E], dtype=np.float64)


class QAOAQtreeSimulator:
    """The reference simulator's energy API over ``QAOAEnergyEngine``."""

    def __init__(self, composer='default', ordering='native', **engine_kw):
        self.engine = QAOAEnergyEngine(composer=composer_name(composer), ordering=ordering, **engine_kw)
        self._distributed = None

    def energy_expectation(self, G, gamma, beta):
        return _reference_shape(G, self.engine.energy_expectation(G, gamma, beta))

    def energy_expectation_parallel(self, G, gamma, beta, n_processes=None):
        return _reference_shape(G, self.engine.energy_expectation(G, gamma, beta))

    def energy_expectation_mpi(self, G, gamma, beta, n_processes=None, print_perf=False):
        import torch.distributed as dist
        if not (dist.is_available() and dist.is_initialized()):
            return _reference_shape(G, self.engine.energy_expectation(G, gamma, beta))
        from .distributed import sharded_energy

        def share(G_, gamma_, beta_, edges):
            return self.engine.energy_expectation(G_, gamma_, beta_, edges=edges)

        return _reference_shape(G, sharded_energy(G, gamma, beta, share, device=self.engine.device))


QAOASimulator = QAOAQtreeSimulator
