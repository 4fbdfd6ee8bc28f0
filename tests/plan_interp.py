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
        idx = tuple(((int(e['sliced_value']) >> a) & 1) if (e['sliced_mask'] >> a) & 1 else slice(None)
                    for a in range(t.ndim))
        kept = [a for a in range(t.ndim) if not (e['sliced_mask'] >> a) & 1]
        t = t[idx]
        perm = [int(x) for x in e['perm'][:e['rank_out']]]
        t = np.transpose(t, [kept.index(a) for a in perm])
        n = 1 << int(e['rank_out'])
        table[e['off']:e['off'] + n] = t.reshape(-1)
    return table


# Shared memory one CTA may use; larger arenas have no chunk tables.
SMEM_LIMIT_BYTES = 224 * 1024


def _pext(x, m):
    """Bit gather on an integer array: the bits of x selected by mask m."""
    x = np.asarray(x, dtype=np.int64)
    r = np.zeros_like(x)
    bit = 0
    for b in range(32):
        if (m >> b) & 1:
            r |= ((x >> b) & 1) << bit
            bit += 1
    return r


def _gather_runs(j, runs):
    """The executor's bit gather from its precompiled runs (None: fallback)."""
    runs = int(runs)
    n = runs >> 60
    if n == 7:
        return None
    if n <= 1:                       # pre-decoded single run
        return (j >> ((runs >> 32) & 31)) & (runs & 0xffffffff)
    off = np.zeros_like(j)
    dst = 0
    for r in range(n):
        rr = (runs >> (10 * r)) & 0x3ff
        start, length = rr & 31, rr >> 5
        off |= ((j >> start) & ((1 << length) - 1)) << dst
        dst += length
    return off


def network_views(exported, net_index):
    """Phases, ops and operands of one network, decoded from its executor
    blob exactly as the device kernel addresses them (network-local)."""
    run = exported['runs'][net_index]
    base = int(run['blob_off16']) * 16
    blob = exported['blobs'][base:base + int(run['blob_bytes'])]
    assert int(run['blob_bytes']) % 16 == 0
    n_ph = int(run['n_phases'])
    ph_bytes = n_ph * _lib.PHASE_DTYPE.itemsize
    phases = blob[:ph_bytes].view(_lib.PHASE_DTYPE)
    ins_off = int(run['ins_off'])
    ops = blob[ph_bytes:ins_off].view(_lib.OP_DTYPE)
    n_ins = int(max([o['in_begin'] + o['k'] for o in ops], default=0))
    ins = blob[ins_off:ins_off + n_ins * _lib.IN_DTYPE.itemsize].view(_lib.IN_DTYPE)
    assert ins_off + n_ins * _lib.IN_DTYPE.itemsize <= len(blob)
    return run, phases, ops, ins


def run_network(exported, table, net_index):
    net, phases, ops, ins = network_views(exported, net_index)
    arena = np.full(int(net['arena_elems']) + 4, np.nan + 0j, dtype=np.complex128)

    def load(src, off):
        if src & _lib.SRC_TABLE:
            base = src & ~_lib.SRC_TABLE
            assert base + off.max() < len(table)
            return table[base + off]
        assert src + off.max() <= int(net['arena_elems'])
        v = arena[src + off]
        assert not np.isnan(v.real).any(), 'read of an arena element nobody wrote'
        return v

    blob = exported['blobs'][int(net['blob_off16']) * 16:
                             int(net['blob_off16']) * 16 + int(net['blob_bytes'])]
    for p in range(int(net['n_phases'])):
        ph = phases[p]
        # the chunk table names the op holding the first element of every
        # 32-element chunk of the phase
        n_chunks = (int(ph['total_elems']) + 31) // 32
        co = int(ph['chunk_off'])
        if 8 * int(net['arena_elems']) > SMEM_LIMIT_BYTES:   # wide: no chunk tables
            assert co == 0
            n_chunks = 0
        assert co + 2 * n_chunks <= len(blob)
        chunks = blob[co:co + 2 * n_chunks].view('<u2')
        starts = ops['elem_begin']
        for c, oi in enumerate(chunks):
            assert int(ph['op_first']) <= oi < int(ph['op_first'] + ph['op_count'])
            e = 32 * c
            assert starts[oi] <= e < starts[oi] + (1 << int(ops[oi]['u'] - ops[oi]['sum']))
        # the executor's op lookup relies on ops of non-increasing size
        widths = [int(ops[o]['u'] - ops[o]['sum'])
                  for o in range(int(ph['op_first']), int(ph['op_first'] + ph['op_count']))]
        assert all(a >= b for a, b in zip(widths, widths[1:]))
        writes = []
        elem = 0
        for o in range(int(ph['op_first']), int(ph['op_first'] + ph['op_count'])):
            op = ops[o]
            u, s, k = int(op['u']), int(op['sum']), int(op['k'])
            w = u - s
            assert op['elem_begin'] == elem
            elem += 1 << w
            operands = ins[int(op['in_begin']):int(op['in_begin']) + k]
            j = np.arange(1 << w, dtype=np.int64)
            acc = np.zeros(1 << w, dtype=np.complex128)
            for sv in range(s + 1):
                prod = np.ones(1 << w, dtype=np.complex128)
                for d in operands:
                    mask = int(d['mask'])
                    off = _pext(j | (sv << w), mask)
                    low = _gather_runs(j, d['runs'])
                    if low is not None:
                        # runs cover the bits below the summed one; the summed
                        # bit is the operand's most significant axis
                        top = (mask >> w) & 1 if s else 0
                        stride = 1 << (bin(mask).count('1') - 1) if top else 0
                        assert np.array_equal(off, low + sv * stride)
                    prod = prod * load(int(d['src']), off)
                acc = acc + prod
            writes.append((int(op['dst']), acc))
        assert elem == ph['total_elems']
        for off, val in writes:          # all reads of a phase precede its writes
            assert off + len(val) <= int(net['arena_elems'])
            arena[off:off + len(val)] = val
    res = int(net['result_src'])
    return table[res & ~_lib.SRC_TABLE] if res & _lib.SRC_TABLE else arena[res]


def run_network_records(exported, table, net_index):
    """A network from its element records, as the shared-memory executor
    reads them: one window S = [gate table, padded to an even length]
    [arena]; every element's output and operand offsets point into S.
    Checks that records cover the phases exactly, that every read hits an
    element written before (or the gate table) and every write the arena."""
    run = exported['runs'][net_index]
    words = int(run['rec_words'])
    assert words > 0
    assert int(run['rec_off']) % 4 == 0       # 16-byte aligned: headers are read as 8-byte pairs
    rec = exported['recs'][int(run['rec_off']):int(run['rec_off']) + words].astype(np.int64)
    n_tab = int(exported['table_elems'])
    pad = (n_tab + 1) & ~1
    arena_elems = int(run['arena_elems'])
    S = np.full(pad + arena_elems, np.nan + 0j, dtype=np.complex128)
    S[:n_tab] = table
    n_ph = int(run['n_phases'])
    used = 2 * n_ph

    def load(off):
        v = S[off]
        assert not np.isnan(v.real).any(), 'read of an element nobody wrote'
        return v

    compact = int(run['rec_format']) == _lib.REC_COMPACT
    if compact:
        assert pad + arena_elems <= 4096
        used = (used + 3) & ~3
    for p in range(n_ph):
        payload, head = int(rec[2 * p]), int(rec[2 * p + 1])
        total, kmax = head & 0xffffff, head >> 24
        assert 1 <= kmax
        if compact:
            # 8 little-endian 16-bit fields per element, decoded into the
            # rows of the wide format
            assert payload % 4 == 0 and kmax <= 7
            f = exported['recs'][int(run['rec_off']) + payload:int(run['rec_off']) + payload + 4 * total]
            f = f.view('<u2').astype(np.int64).reshape(total, 8)
            used += 4 * total
            d = f[:, 0]
            k = ((d >> 12) & 7) + 1
            assert np.all(k <= kmax)
            rows = np.zeros((kmax + 1, total), dtype=np.int64)
            rows[0] = (d & 0xfff) | k << 16 | (d >> 15) << 24
            for t in range(kmax):
                o0 = f[:, 1 + t] & 0xfff
                code = f[:, 1 + t] >> 12
                o1 = o0 + ((1 << code) >> 1)
                assert np.all((f[:, 1 + t] == 0) | (t < k))
                rows[1 + t] = np.where(t < k, o0 | o1 << 16, 0)
        else:
            rows = rec[payload:payload + (kmax + 1) * total].reshape(kmax + 1, total)
            used += (kmax + 1) * total
        d = rows[0]
        dst, k, s = d & 0xffff, (d >> 16) & 0xff, d >> 24
        assert np.all((k >= 1) & (k <= kmax)) and np.all((s == 0) | (s == 1))
        assert np.all((dst >= pad) & (dst < pad + arena_elems))
        assert len(np.unique(dst)) == total
        p0 = load(rows[1] & 0xffff)
        p1 = load(rows[1] >> 16)
        for t in range(2, kmax + 1):
            live = t <= k
            lo, hi = rows[t][live] & 0xffff, rows[t][live] >> 16
            p0[live] = p0[live] * load(lo)
            p1[live] = p1[live] * load(hi)
        S[dst] = np.where(s == 1, p0 + p1, p0)
    assert used == words
    res = int(run['result_src'])
    return table[res & ~_lib.SRC_TABLE] if res & _lib.SRC_TABLE else S[pad + res]


def run_plan(plan, params, per_circuit=True, records=False):
    """Amplitude of every circuit (slices summed), or of every network;
    with ``records`` every network that has element records is run from
    them."""
    ex = plan.export()
    table = gate_table(ex, np.asarray(params, dtype=np.float64))
    vals = np.array([run_network_records(ex, table, i) if records and ex['runs'][i]['rec_words']
                     else run_network(ex, table, i) for i in range(len(ex['runs']))])
    if not per_circuit:
        return vals
    groups = plan.groups()
    out = np.zeros(groups.max() + 1 if len(groups) else 0, dtype=np.complex128)
    np.add.at(out, groups, vals)
    return out
