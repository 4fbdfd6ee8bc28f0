"""Clean-room CPU restatement of the ``qtree`` package subset that QTensor's
bucket-elimination path calls.  TEST INFRASTRUCTURE ONLY: nothing in the
``qtensor_b200`` product may import this package; only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it, and
only as the checker / the timed reference implementation.

Third-party boundary
--------------------
QTensor imports ``qtree`` (github.com/DaniloZZZ/qtree, PyPI ``qtensor-qtree``)
as a git submodule (``.gitmodules:1-3``) that is empty in the reference
checkout, and ``setup.py:16`` depends on ``qtensor-qtree`` with **no version
pin**.  This package restates the published algorithm of that dependency from
the behaviour QTensor's own call sites document:

* ``qtensor/ProcessingFrameworks.py:29-37, 45-147`` -- bucket semantics
  (sorted-union indices, sum over the first index, ``E<tag>`` naming, the
  ``no_sum`` branch, tag ``'f'`` for scalars);
* ``qtensor/Simulate.py:47-58, 90-94`` -- reorder by peo, slicing of bra/ket
  variables, ``bucket_elimination(..., n_var_nosum)``;
* ``qtensor/FeynmanSimulator.py:18-25, 49-58`` -- integer slicing and the
  ``unravel_index`` helper;
* ``qtensor/optimisation/*.py`` -- line-graph node attributes ``name`` and
  ``size``; ``make_clique_on`` / ``get_equivalent_peo``;
* ``examples/scripts_jupytext/Basic usage.py:48-195`` -- ``circ2buckets``
  layout (bra first, ket measurement tensors in ``buckets[-2]`` for one qubit),
  ``slice_from_bits`` and the need to reorder before eliminating;
* ``qtensor/OpFactory.py:31-60`` -- ``ParametricGate`` / ``gen_tensor`` /
  ``parameters`` / ``LABEL_TO_GATE_DICT``; gate conventions pinned physically
  by ``qtensor/tests/test_qaoa_energy.py:58`` and
  ``qtensor/tests/qiskit_qaoa_energy.py:107``;
* ``qtensor/simplify_circuit/simplify_circuit_api.py:85-104`` -- daggered gates
  keep their class, carry ``'+'`` in ``name`` and the original ``alpha``.

Parity with the real (unpinned) qtree is therefore anchored on those call
sites plus independent physics oracles (dense state vector, the analytic p=1
QAOA edge formula, the Petersen p=9 known answer of
``qtensor/tests/qiskit_qaoa_energy.py:112-123``).
"""
from . import optimizer
from . import operators
from . import operators_full_matrix
from . import np_framework
from . import utils
from . import graph_model

__all__ = ['optimizer', 'operators', 'operators_full_matrix', 'np_framework',
           'utils', 'graph_model']
