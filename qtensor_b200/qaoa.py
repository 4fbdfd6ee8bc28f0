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
"""
from .engine import QAOAEnergyEngine

_COMPOSERS = {'DefaultQAOAComposer': 'default', 'ZZQtreeQAOAComposer': 'zz',
              'QtreeQAOAComposer': 'cx', 'default': 'default', 'zz': 'zz', 'cx': 'cx'}


def composer_name(composer):
    key = composer if isinstance(composer, str) else getattr(composer, '__name__', type(composer).__name__)
    if key not in _COMPOSERS:
        raise ValueError('composer {!r} is not supported'.format(key))
    return _COMPOSERS[key]


class QAOAQtreeSimulator:
    """The reference simulator's energy API over ``QAOAEnergyEngine``."""

    def __init__(self, composer='default', ordering='native', **engine_kw):
        self.engine = QAOAEnergyEngine(composer=composer_name(composer), ordering=ordering, **engine_kw)
        self._distributed = None

    def energy_expectation(self, G, gamma, beta):
        return self.engine.energy_expectation(G, gamma, beta)

    def energy_expectation_parallel(self, G, gamma, beta, n_processes=None):
        return self.engine.energy_expectation(G, gamma, beta)

    def energy_expectation_mpi(self, G, gamma, beta, n_processes=None, print_perf=False):
        import torch.distributed as dist
        if not (dist.is_available() and dist.is_initialized()):
            return self.engine.energy_expectation(G, gamma, beta)
        from .distributed import sharded_energy

        def share(G_, gamma_, beta_, edges):
            return self.engine.energy_expectation(G_, gamma_, beta_, edges=edges)

        return sharded_energy(G, gamma, beta, share, device=self.engine.device)


QAOASimulator = QAOAQtreeSimulator
