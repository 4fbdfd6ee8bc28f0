"""Variables, tensors, circuit -> buckets, reordering and bucket elimination.

Oracle restatement of the ``qtree.optimizer`` API used by QTensor
(``qtensor/Simulate.py:48,90``, ``qtensor/FeynmanSimulator.py:54``,
``qtensor/optimisation/TensorNet.py:65``, ``qtensor/ProcessingFrameworks.py:96,146``).
Test infrastructure only.
"""
import numbers

from . import operators as ops


class Var:
    """A binary (in general ``size``-valued) contraction index.

    QTensor relies on ``int(var)`` being the identity, on ``.size``, ``.name``
    and ``.identity`` (``qtensor/optimisation/Optimizer.py:33-35,60-62``,
    ``qtensor/ProcessingFrameworks.py:87``) and on sorting by ``int``.
    """
    __slots__ = ('_identity', '_size', '_name', '_hash')

    def __init__(self, identity, size=2, name=None):
        if not isinstance(identity, numbers.Integral):
            raise ValueError('Var identity must be an integer, got {!r}'.format(identity))
        self._identity = int(identity)
        self._size = int(size)
        self._name = name if name is not None else 'v_{}'.format(int(identity))
        self._hash = hash((self._identity, self._name, self._size))

    @property
    def identity(self):
        return self._identity

    @property
    def size(self):
        return self._size

    @property
    def name(self):
        return self._name

    def copy(self, identity=None, size=None, name=None):
        """New index; a new identity gets the default name unless ``name`` is given."""
        if identity is None:
            identity = self._identity
            if name is None:
                name = self._name
        if size is None:
            size = self._size
        return Var(identity, size=size, name=name)

    def __int__(self):
        return self._identity

    def __index__(self):
        return self._identity

    def __hash__(self):
        return self._hash

    def __eq__(self, other):
        return (isinstance(other, Var) and self._identity == other._identity
                and self._size == other._size and self._name == other._name)

    def __lt__(self, other):
        return self._identity < int(other)

    def __str__(self):
        return self._name

    __repr__ = __str__

    def __getstate__(self):
        return (self._identity, self._size, self._name)

    def __setstate__(self, state):
        self._identity, self._size, self._name = state
        self._hash = hash((self._identity, self._name, self._size))


class Tensor:
    """A named tensor over ``indices``; its array is ``data`` or ``data_dict[data_key]``."""

    def __init__(self, name, indices, data_key=None, data=None):
        self._name = name
        self._indices = tuple(indices)
        self._data_key = data_key
        self._data = data

    @property
    def name(self):
        return self._name

    @property
    def indices(self):
        return self._indices

    @property
    def shape(self):
        return tuple(v.size for v in self._indices)

    @property
    def data_key(self):
        return self._data_key

    @property
    def data(self):
        return self._data

    def copy(self, name=None, indices=None, data_key=None, data=None):
        return Tensor(self._name if name is None else name,
                      self._indices if indices is None else indices,
                      self._data_key if data_key is None else data_key,
                      self._data if data is None else data)

    def __mul__(self, other):
        """Product used by ``bucket_elimination`` to fold scalar results."""
        if self._data is None or other._data is None:
            raise ValueError('cannot multiply tensors without data')
        if len(other._indices) == 0:
            return self.copy(data=self._data * other._data)
        if len(self._indices) == 0:
            return other.copy(data=self._data * other._data)
        if self._indices != other._indices:
            raise ValueError('product of tensors with different indices: '
                             '{} vs {}'.format(self._indices, other._indices))
        return self.copy(data=self._data * other._data)

    def __str__(self):
        return '{}({})'.format(self._name, ','.join(map(str, self._indices)))

    __repr__ = __str__


def _data_key(op):
    return (op.name, tuple(sorted(op.parameters.items())))


def circ2buckets(qubit_count, circuit, pdict=None, max_depth=None):
    """Build the bucket representation of ``<bra| circuit |ket>``.

    Layout (``examples/scripts_jupytext/Basic usage.py:48-110``):

    * variables ``0..qubit_count-1`` are the bra (output) indices ``o_q``;
    * the network is built from the bra side backwards: a measurement tensor
      ``M`` on every qubit, then the gates in reverse order;
    * a gate whose qubit is in ``changed_qubits`` gets the pair
      ``(current frame var, new var)`` for that qubit, other qubits only the
      current frame var (diagonal gates create no variables);
    * every tensor goes to the bucket of its smallest variable;
    * finally a measurement tensor ``(frame var, i_q)`` closes every qubit;
      ``i_q`` are the ket (input) indices.

    Returns ``(buckets, data_dict, bra_variables, ket_variables)``.
    """
    if max_depth is None:
        max_depth = len(circuit)
    data_dict = {}
    frame = [Var(q, name='o_{}'.format(q)) for q in range(qubit_count)]
    bra_variables = list(frame)
    next_id = qubit_count
    buckets = [[] for _ in range(qubit_count)]

    layers = [[ops.M(q) for q in range(qubit_count)]]
    layers += list(reversed(circuit[:max_depth]))
    for layer in layers:
        for op in layer:
            changed = set(op.changed_qubits)
            indices = []
            new_id = next_id
            for q in op.qubits:
                indices.append(frame[q])
                if q in changed:
                    indices.append(Var(new_id))
                    new_id += 1
            key = _data_key(op)
            if key not in data_dict:
                data_dict[key] = ops.gate_tensor(op)
            smallest = min(int(v) for v in indices)
            buckets[smallest].append(Tensor(op.name, indices, data_key=key))
            for q in op.qubits:
                if q in changed:
                    frame[q] = Var(next_id)
                    buckets.append([])
                    next_id += 1

    ket_variables = []
    m = ops.M(0)
    key = _data_key(m)
    data_dict[key] = ops.gate_tensor(m)
    for q in range(qubit_count):
        var = frame[q]
        ket = Var(next_id, name='i_{}'.format(q))
        ket_variables.append(ket)
        buckets[int(var)].append(Tensor(m.name, [var, ket], data_key=key))
        buckets.append([])
        frame[q] = ket
        next_id += 1
    return buckets, data_dict, bra_variables, ket_variables


def reorder_buckets(old_buckets, permutation):
    """Relabel variables so ``permutation[n]`` becomes identity ``n`` and
    redistribute tensors to the bucket of their (new) smallest index
    (``qtensor/Simulate.py:47-52``).  Default-named (``v_*``) variables take the
    new default name; named ones (``o_*``, ``i_*``) keep theirs.
    Returns ``(new_buckets, perm_dict)``.
    """
    perm_dict = {}
    for n, var in enumerate(permutation):
        if var.name.startswith('v'):
            perm_dict[var] = var.copy(n)
        else:
            perm_dict[var] = var.copy(n, name=var.name)
    new_buckets = [[] for _ in range(len(old_buckets))]
    for bucket in old_buckets:
        for tensor in bucket:
            new_indices = [perm_dict[v] for v in tensor.indices]
            target = min(int(v) for v in new_indices)
            new_buckets[target].append(tensor.copy(indices=new_indices))
    return new_buckets, perm_dict


def bucket_elimination(buckets, process_bucket_fn, n_var_nosum=0):
    """Eliminate buckets in order (``qtensor/Simulate.py:90-93``).

    Each non-empty bucket among the first ``len(buckets) - n_var_nosum`` is
    processed with summation; a non-scalar result is appended to the bucket of
    its first (smallest) index, scalar results are multiplied together.  The
    tensors of the last ``n_var_nosum`` buckets are multiplied without
    summation (``process_bucket_fn(rest, no_sum=True)``).
    """
    result = None
    n_sum = len(buckets) - n_var_nosum
    for bucket in buckets[:n_sum]:
        if len(bucket) == 0:
            continue
        tensor = process_bucket_fn(bucket)
        if len(tensor.indices) > 0:
            buckets[int(tensor.indices[0])].append(tensor)
        else:
            result = tensor if result is None else result * tensor
    rest = [t for bucket in buckets[n_sum:] for t in bucket]
    if rest:
        tensor = process_bucket_fn(rest, no_sum=True)
        result = tensor if result is None else result * tensor
    return result
