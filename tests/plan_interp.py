"""CPU interpreter of exported ``qtb_plan`` arrays (test infrastructure).

Executes the plan exactly as the device executor does (phases, ops, operand
masks, arena offsets, gate-table entries) but in complex128 numpy, with the
gate tensors taken from the oracle's qtree operators.  Checks the C++ plan
compiler on machines without a GPU.
"""
import numpy as np

from qtensor_b200 import _lib

import qtree.operators as qops
import qtensor_port


def _gate_tensor(kind, alpha):
    k = kind
    if k == _lib.GATE_M:
        return qops.M(0).gen_tensor()
    if k == _lib.GATE_H:
        return qops.H(0).gen_tensor()
    if k == _lib.GATE_Z:
        return qops.Z(0).gen_tensor()
    if k == _lib.GATE_X:
        return qops.X(0).gen_tensor()
    if k == _lib.GATE_Y:
        return qops.Y(0).gen_tensor()
    if k == _lib.GATE_T:
        return qops.T(0).gen_tensor()
    if k == _lib.GATE_CX:
        return qops.cX(0, 1).gen_tensor()
    if k == _lib.GATE_CZ:
        return qops.cZ(0, 1).gen_tensor()
    if k == _lib.GATE_ZPHASE:
        return qops.ZPhase(0, alpha=alpha).gen_tensor()
    if k == _lib.GATE_XPHASE:
        return qops.XPhase(0, alpha=alpha).gen_tensor()
    if k == _lib.GATE_YPHASE:
        return qops.YPhase(0, alpha=alpha).gen_tensor()
    if k == _lib.GATE_ZZ:
        return qtensor_port.ZZ(0, 1, alpha=alpha).gen_tensor()
    raise ValueError(kind)


def gate_table(exported, params):
    """Complex128 gate table for ``params`` (layout of the device table)."""
    table = np.zeros(exported['table_elems'], dtype=np.complex128)
    terms = exported['terms']
    for e in exported['entries']:
        alpha = sum(terms[i]['coef'] * params[terms[i]['param']]
                    for i in range(e['expr_begin'], e['expr_begin'] + e['expr_count']))
        t = np.asarray(_gate_tensor(int(e['kind']), alpha), dtype=np.complex128)
        assert t.ndim == e['rank_in']
        idx = tuple(0 if (e['sliced_mask'] >> a) & 1 else slice(None) for a in range(t.ndim))
        kept = [a for a in range(t.ndim) if not (e['sliced_mask'] >> a) & 1]
        t = t[idx]
        perm = [int(x) for x in e['perm'][:e['rank_out']]]
        t = np.transpose(t, [kept.index(a) for a in perm])
        n = 1 << int(e['rank_out'])
        table[e['off']:e['off'] + n] = t.reshape(-1)
    return table


def _pext(x, m):
    r, bit = 0, 1
    while m:
        low = m & -m
        if x & low:
            r |= bit
        bit <<= 1
        m ^= low
    return r


def run_network(exported, table, net_index):
    net = exported['nets'][net_index]
    ops, ins, phases = exported['ops'], exported['ins'], exported['phases']
    arena = np.full(int(net['arena_elems']) + 4, np.nan + 0j, dtype=np.complex128)

    def load(src, off):
        if src & _lib.SRC_TABLE:
            return table[(src & ~_lib.SRC_TABLE) + off]
        v = arena[src + off]
        assert not np.isnan(v.real), 'read of an arena element nobody wrote'
        return v

    for p in range(int(net['phase_begin']), int(net['phase_begin'] + net['n_phases'])):
        ph = phases[p]
        writes = []
        elem = 0
        for o in range(int(ph['op_first']), int(ph['op_first'] + ph['op_count'])):
            op = ops[o]
            u, s, k = int(op['u']), int(op['sum']), int(op['k'])
            w = u - s
            assert op['elem_begin'] == elem
            elem += 1 << w
            operands = ins[int(op['in_begin']):int(op['in_begin']) + k]
            for j in range(1 << w):
                acc = 0j
                for sv in range(s + 1):
                    idx = j | (sv << w)
                    prod = 1 + 0j
                    for d in operands:
                        prod *= load(int(d['src']), _pext(idx, int(d['mask'])))
                    acc += prod
                writes.append((int(op['dst']) + j, acc))
        assert elem == ph['total_elems']
        for off, val in writes:          # all reads of a phase precede its writes
            arena[off] = val
    res = int(net['result_src'])
    return table[res & ~_lib.SRC_TABLE] if res & _lib.SRC_TABLE else arena[res]


def run_plan(plan, params):
    ex = plan.export()
    table = gate_table(ex, np.asarray(params, dtype=np.float64))
    return np.array([run_network(ex, table, i) for i in range(len(ex['nets']))])
